// Device-side math shared by the baking_b200 kernels (sm_100a).
//
// Per-particle physics of the reference kernels as __device__ functions, so the
// one-kernel-per-reference-kernel entry points and the fused substep kernels run
// the same arithmetic. Precision follows the reference: float32 where its Warp
// kernel uses `float`, float64 where it uses `wp.float64`.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define BK_DEV __device__ __forceinline__

namespace bk {

struct M3 { float m[9]; };
struct M3d { double m[9]; };
struct V3 { float v[3]; };

// ------------------------------------------------------------- SoA access
BK_DEV V3 load_v3(const float* __restrict__ p, int64_t i, int64_t pitch) {
    V3 r;
#pragma unroll
    for (int c = 0; c < 3; ++c) r.v[c] = __ldg(p + c * pitch + i);
    return r;
}
BK_DEV void store_v3(float* __restrict__ p, int64_t i, int64_t pitch, const V3& a) {
#pragma unroll
    for (int c = 0; c < 3; ++c) p[c * pitch + i] = a.v[c];
}
BK_DEV M3 load_m3(const float* __restrict__ p, int64_t i, int64_t pitch) {
    M3 r;
#pragma unroll
    for (int c = 0; c < 9; ++c) r.m[c] = __ldg(p + c * pitch + i);
    return r;
}
BK_DEV void store_m3(float* __restrict__ p, int64_t i, int64_t pitch, const M3& a) {
#pragma unroll
    for (int c = 0; c < 9; ++c) p[c * pitch + i] = a.m[c];
}

// ------------------------------------------------------------- 3x3 algebra
BK_DEV float det3(const M3& a) {
    const float* m = a.m;
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
BK_DEV double det3(const M3d& a) {
    const double* m = a.m;
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6])
         + m[2] * (m[3] * m[7] - m[4] * m[6]);
}
BK_DEV M3 matmul(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
    return r;
}
// Adjugate / determinant.
BK_DEV M3 inverse3(const M3& a) {
    const float* m = a.m;
    float inv = 1.0f / det3(a);
    M3 r;
    r.m[0] = (m[4] * m[8] - m[5] * m[7]) * inv;
    r.m[1] = (m[2] * m[7] - m[1] * m[8]) * inv;
    r.m[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    r.m[3] = (m[5] * m[6] - m[3] * m[8]) * inv;
    r.m[4] = (m[0] * m[8] - m[2] * m[6]) * inv;
    r.m[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    r.m[6] = (m[3] * m[7] - m[4] * m[6]) * inv;
    r.m[7] = (m[1] * m[6] - m[0] * m[7]) * inv;
    r.m[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
    return r;
}

// 3x3 SVD A = U diag(s) V^T in float64 by one-sided Jacobi (Hestenes 1958): right
// plane rotations orthogonalise A's columns; column norms are the singular values.
BK_DEV void svd3(const M3d& A, M3d& U, double s[3], M3d& V) {
    double b[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) b[e] = A.m[e];
    double v[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int sweep = 0; sweep < 40; ++sweep) {
        bool rotated = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int p = k == 2 ? 1 : 0;
            const int q = k == 0 ? 1 : 2;
            double alpha = 0, beta = 0, gamma = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                alpha += b[3 * r + p] * b[3 * r + p];
                beta += b[3 * r + q] * b[3 * r + q];
                gamma += b[3 * r + p] * b[3 * r + q];
            }
            if (gamma == 0.0 || fabs(gamma) <= 1e-15 * sqrt(alpha * beta)) continue;
            rotated = true;
            double zeta = (beta - alpha) / (2.0 * gamma);
            double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            double c = rsqrt(1.0 + t * t);
            double sn = c * t;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                double bp = b[3 * r + p], bq = b[3 * r + q];
                b[3 * r + p] = c * bp - sn * bq;
                b[3 * r + q] = sn * bp + c * bq;
                double vp = v[3 * r + p], vq = v[3 * r + q];
                v[3 * r + p] = c * vp - sn * vq;
                v[3 * r + q] = sn * vp + c * vq;
            }
        }
        if (!rotated) break;
    }
    bool zero[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double n = sqrt(b[c] * b[c] + b[3 + c] * b[3 + c] + b[6 + c] * b[6 + c]);
        s[c] = n;
        zero[c] = !(n > 1e-300);
        double inv = zero[c] ? 0.0 : 1.0 / n;
#pragma unroll
        for (int r = 0; r < 3; ++r) U.m[3 * r + c] = b[3 * r + c] * inv;
    }
    if (zero[0] || zero[1] || zero[2]) {
        // Rank-deficient input: complete U to an orthonormal basis.
        for (int c = 0; c < 3; ++c) {
            if (!zero[c]) continue;
            int a = (c + 1) % 3, d = (c + 2) % 3;
            double ua[3] = {U.m[a], U.m[3 + a], U.m[6 + a]}, ud[3] = {U.m[d], U.m[3 + d], U.m[6 + d]};
            if (zero[a]) {
                ua[0] = fabs(ud[0]) < 0.9 ? 1.0 : 0.0;
                ua[1] = 1.0 - ua[0];
                ua[2] = 0.0;
                double dp = ua[0] * ud[0] + ua[1] * ud[1] + ua[2] * ud[2];
                for (int r = 0; r < 3; ++r) ua[r] -= dp * ud[r];
                double n = sqrt(ua[0] * ua[0] + ua[1] * ua[1] + ua[2] * ua[2]);
                for (int r = 0; r < 3; ++r) { ua[r] /= n; U.m[3 * r + a] = ua[r]; }
                zero[a] = false;
            }
            U.m[c] = ua[1] * ud[2] - ua[2] * ud[1];
            U.m[3 + c] = ua[2] * ud[0] - ua[0] * ud[2];
            U.m[6 + c] = ua[0] * ud[1] - ua[1] * ud[0];
            zero[c] = false;
        }
    }
#pragma unroll
    for (int e = 0; e < 9; ++e) V.m[e] = v[e];
}

// ------------------------------------------------- physics/transfer.py:4-28
BK_DEV float qweight(float l, int i) {
    if (i == 0) return 0.5f * (1.5f - l) * (1.5f - l);
    if (i == 1) return 0.75f - (l - 1.0f) * (l - 1.0f);
    return 0.5f * (l - 0.5f) * (l - 0.5f);
}

struct Stencil {
    int b[3];
    float l[3];
    float w[3][3];  // w[axis][offset]
    bool valid;
};

BK_DEV Stencil make_stencil(const V3& x, const float* origin, float dx, int R) {
    Stencil s;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float g = (x.v[a] - origin[a]) / dx;
        s.b[a] = (int)floorf(g - 0.5f);
        s.l[a] = g - (float)s.b[a];
    }
    s.valid = s.b[0] >= 0 && s.b[1] >= 0 && s.b[2] >= 0 && s.b[0] + 2 < R && s.b[1] + 2 < R && s.b[2] + 2 < R;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int o = 0; o < 3; ++o) s.w[a][o] = qweight(s.l[a], o);
    return s;
}

BK_DEV int64_t node_index(int i, int j, int k, int R) { return ((int64_t)i * R + j) * R + k; }

BK_DEV void set_flag(int32_t* flags, int index) {
    if (flags[index] == 0) atomicMax(flags + index, 1);
}

// ------------------------------------------------------- ding.py:56-100
BK_DEV float temperature_factor(float T, const float* knots, const float* factors) {
    float f = factors[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (T >= knots[k]) {
            float frac = fminf((T - knots[k]) / (knots[k + 1] - knots[k]), 1.0f);
            f = (1.0f - frac) * factors[k] + frac * factors[k + 1];
        }
    }
    return f;
}

BK_DEV float porosity_coefficient(float n) {
    float c = 0.0f;
    if (n > 0.0f) {
        float lg = logf(1.0f / n);
        c = 9.0f / (4.0f * (lg * lg) * (3.5f * n + 1.0f));
    }
    return c;
}

// Scalar overstress Newton solve (ding.py:77-87): 32 steps from r = 0 in float32.
// Iterates of this concave increasing residual approach the root monotonically from
// below, so once a step no longer changes r the remaining steps are no-ops.
BK_DEV float solve_overstress(float q2, float p2, float d, float h) {
    float r = 0.0f;
    if (q2 + p2 > 1.0f) {
        for (int it = 0; it < 32; ++it) {
            float dd = 1.0f + d * r, md = 1.0f + h * r;
            float dd2 = dd * dd, md2 = md * md;
            float res = r + 1.0f - q2 / dd2 - p2 / md2;
            float der = 1.0f + 2.0f * d * q2 / (dd2 * dd) + 2.0f * h * p2 / (md2 * md);
            float rn = r - res / der;
            if (rn == r) break;
            r = rn;
        }
    }
    return r;
}

// --------------------------------------- porous_return.py:11-61 (float64)
BK_DEV double pressure_coefficient64(double n) {
    double c = 0.0;
    if (n > 0.0) {
        double lg = log(1.0 / n);
        c = 9.0 / (4.0 * (lg * lg) * (3.5 * n + 1.0));
    }
    return c;
}

BK_DEV double overstress64(double q, double p, double d, double h) {
    double r = 0.0;
    if (q + p > 1.0) {
        for (int it = 0; it < 48; ++it) {
            double u = 1.0 + d * r, v = 1.0 + h * r;
            double u2 = u * u, v2 = v * v;
            double res = r + 1.0 - q / u2 - p / v2;
            double der = 1.0 + 2.0 * d * q / (u2 * u) + 2.0 * h * p / (v2 * v);
            r -= res / der;
            if (fabs(res) < 1.0e-12) break;
        }
    }
    return r;
}

BK_DEV double porosity_prediction(double n, float q, float p, float d, float h, float e, double Vp, float n0) {
    double a = pressure_coefficient64(n);
    double r = overstress64((double)q, a * (double)p, (double)d, (double)h * a);
    double den = 1.0 + (double)h * a * r;
    return Vp * exp((double)e * (1.0 - 1.0 / den)) - 1.0 + (double)n0;
}

// End-state porosity (porous_return.py:43-61): elastic early exit, else 64 bisection
// steps of n -> prediction(n) on [0, 1 - 1e-9].
BK_DEV float solve_porosity(float q, float p, float d, float h, float e, double Vp, float n0) {
    double trial = Vp - 1.0 + (double)n0;
    if (trial > 0.0 && trial < 1.0) {
        double a = pressure_coefficient64(trial);
        if ((double)q + a * (double)p <= 1.0) return (float)trial;
    }
    double lo = 0.0, hi = 1.0 - 1.0e-9;
    for (int it = 0; it < 64; ++it) {
        double mid = (lo + hi) * 0.5;
        double pred = porosity_prediction(mid, q, p, d, h, e, Vp, n0);
        if (mid < pred) lo = mid; else hi = mid;
    }
    return (float)((lo + hi) * 0.5);
}

struct DingOut {
    M3 Fe, tau;
    float residual;
};

// Ding return map (ding.py:103-137) given the float64 SVD of the trial gradient.
BK_DEV DingOut ding_return(const M3& trial, const M3d& Ud, const double* sd, const M3d& Vd, float mu, float lam,
                           float ty, float eta, float a, float dt) {
    float U[9], V[9], s[3];
#pragma unroll
    for (int e = 0; e < 9; ++e) { U[e] = (float)Ud.m[e]; V[e] = (float)Vd.m[e]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) s[k] = (float)sd[k];
    float eps[3] = {logf(s[0]), logf(s[1]), logf(s[2])};
    float tr = eps[0] + eps[1] + eps[2];
    float ts[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * eps[k] + lam * tr;
    float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
    float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
    float ty2 = ty * ty;
    float q2 = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / ty2;
    float p2 = a * mean * mean / ty2;
    float df = 6.0f * mu * dt * ty * ty / eta;
    float mf = 2.0f * a / 3.0f * (2.0f * mu + 3.0f * lam) * dt * ty * ty / eta;
    float r = solve_overstress(q2, p2, df, mf);
    float cs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) cs[k] = dev[k] / (1.0f + df * r) + mean / (1.0f + mf * r);
    float cm = (cs[0] + cs[1] + cs[2]) / 3.0f;
    float ex[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ex[k] = expf((cs[k] - cm) / (2.0f * mu) + cm / (2.0f * mu + 3.0f * lam));
    DingOut o;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            o.Fe.m[3 * i + k] = (U[3 * i] * ex[0]) * V[3 * k] + (U[3 * i + 1] * ex[1]) * V[3 * k + 1]
                              + (U[3 * i + 2] * ex[2]) * V[3 * k + 2];
            o.tau.m[3 * i + k] = (U[3 * i] * cs[0]) * U[3 * k] + (U[3 * i + 1] * cs[1]) * U[3 * k + 1]
                               + (U[3 * i + 2] * cs[2]) * U[3 * k + 2];
        }
    if (a == 0.0f) {
        float scale = powf(det3(trial) / det3(o.Fe), 1.0f / 3.0f);
#pragma unroll
        for (int e = 0; e < 9; ++e) o.Fe.m[e] *= scale;
    }
    o.residual = 0.0f;
    if (q2 + p2 > 1.0f) {
        float u = 1.0f + df * r, w = 1.0f + mf * r;
        o.residual = fabsf(r + 1.0f - q2 / (u * u) - p2 / (w * w));
    }
    return o;
}

struct DingParamsDev {
    int coupled_porosity, temperature_enabled;
    float mu, lam, yield_stress, initial_porosity, dt;
    float knots[4], yield_factors[4], viscosity_factors[4];
};

struct DingParticleOut {
    M3 Fe, Fp, tau;
    float residual, porosity, porosity_residual, yield_stress, viscosity;
    int gelled;
};

// UpdateDing for one particle (ding.py:154-221). Returns false when the old porosity is
// outside [0, 1) (flag 0 set, nothing written, as in the reference).
BK_DEV bool update_ding_particle(const DingParamsDev& P, const M3& Fe_old, float por, int gel, const M3& F_tot,
                                 const M3& C_new, float T, float eta_base, int32_t* flags, DingParticleOut& out) {
    if (!isfinite(por) || por < 0.0f || por >= 1.0f) { set_flag(flags, 0); return false; }
    int reached = T >= P.knots[3];
    float Teff = T;
    float ty = P.yield_stress;
    float eta = eta_base;
    if (P.temperature_enabled) {
        if (reached) gel = 1;
        if (gel) Teff = P.knots[3];
        ty = P.yield_stress * temperature_factor(Teff, P.knots, P.yield_factors);
        eta = eta_base * temperature_factor(Teff, P.knots, P.viscosity_factors);
    }
    const float dt = P.dt, mu = P.mu, lam = P.lam, n0 = P.initial_porosity;
    M3 G = C_new;
#pragma unroll
    for (int e = 0; e < 9; ++e) G.m[e] = dt * C_new.m[e] + ((e % 4) == 0 ? 1.0f : 0.0f);
    M3 trial = matmul(G, Fe_old);
    M3d Ad, Ud, Vd;
    double sd[3];
#pragma unroll
    for (int e = 0; e < 9; ++e) Ad.m[e] = (double)trial.m[e];
    svd3(Ad, Ud, sd, Vd);
    float ret_por = por, consistency = 0.0f;
    if (P.coupled_porosity) {
        float st[3] = {logf((float)sd[0]), logf((float)sd[1]), logf((float)sd[2])};
        float tr = st[0] + st[1] + st[2];
        float ts[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * st[k] + lam * tr;
        float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
        float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
        float ty2 = ty * ty;
        float qv = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / ty2;
        float pv = mean * mean / ty2;
        float df = 6.0f * mu * dt * ty * ty / eta;
        float ms = 2.0f / 3.0f * (2.0f * mu + 3.0f * lam) * dt * ty * ty / eta;
        float ex = 3.0f * mean / (2.0f * mu + 3.0f * lam);
        double Vp = 1.0 - (double)n0 + (double)por;
        ret_por = solve_porosity(qv, pv, df, ms, ex, Vp, n0);
        double pred = porosity_prediction((double)ret_por, qv, pv, df, ms, ex, Vp, n0);
        consistency = (float)fabs((double)ret_por - pred);
        if (consistency > 1.0e-6f || ret_por <= 0.0f || ret_por >= 1.0f) set_flag(flags, 1);
    }
    DingOut d = ding_return(trial, Ud, sd, Vd, mu, lam, ty, eta, porosity_coefficient(ret_por), dt);
    M3 Fe = d.Fe;
    if (P.coupled_porosity) {
        double target = 1.0 - (double)n0 + (double)ret_por;
        M3d Fd, Fed;
#pragma unroll
        for (int e = 0; e < 9; ++e) { Fd.m[e] = (double)F_tot.m[e]; Fed.m[e] = (double)Fe.m[e]; }
        double vs = det3(Fd) / (target * det3(Fed));
        float scale = (float)pow(vs, 1.0 / 3.0);
#pragma unroll
        for (int e = 0; e < 9; ++e) Fe.m[e] *= scale;
    }
    M3 Fp = matmul(inverse3(Fe), F_tot);
    float npor = det3(Fp) - 1.0f + n0;
    if (P.coupled_porosity) npor = ret_por;
    if (n0 == 0.0f && por == 0.0f) npor = 0.0f;
    if (!isfinite(npor) || npor < 0.0f || npor >= 1.0f) set_flag(flags, 0);
    out.Fe = Fe;
    out.Fp = Fp;
    out.tau = d.tau;
    out.residual = d.residual;
    out.porosity = npor;
    out.porosity_residual = consistency;
    out.yield_stress = ty;
    out.viscosity = eta;
    out.gelled = gel;
    return true;
}

// --------------------------------------------------- gas.py:7-13
constexpr double kGasConstant = 8.31446261815324;

BK_DEV double gas_pressure(double moles, float T, float J, float n) {
    return moles * kGasConstant * (double)T / ((double)J * (double)n);
}

}  // namespace bk
