// Hand-written adjoint of the mechanics substep (P2G -> grid update -> G2P -> return map).
//
// Reverse order of one substep t -> t+1, given the adjoint of state t+1 and the forward grid of step
// t (node mass, momentum and velocity, recomputed by the caller from the checkpointed state t):
//
//   adj_g2p_return   per particle: recompute G2P and the return map, then pull the adjoints of
//                    v', C', F', Fe', tau', porosity' back to F, Fe, porosity, temperature and the
//                    material parameters, and form the v-bar, C-bar the G2P gather receives.
//   adj_g2p_scatter  per particle: the weight-gradient terms of x; v-bar, C-bar scattered to the
//                    grid-velocity adjoint through shared-memory tiles (the forward P2G's scheme).
//   adj_grid         per node: velocity adjoint -> momentum and mass adjoints (walls clamp to zero).
//   adj_p2g          per particle: gather the momentum/mass adjoints -> v, C, tau (and, for the
//                    neo-Hookean model, F and mu, lambda) and the weight-gradient terms of x.
//
// The return map's backward uses the derivative of isotropic matrix functions: with trial
// A = U diag(s) V^T, Fe' = U diag(g(s)) V^T and tau' = U diag(h(s)) U^T, the off-diagonal terms
// in the rotated frame use divided differences of g and h. For this model they have closed
// forms (g_j - g_i and h_j - h_i depend on log(s_j / s_i) alone), evaluated with expm1/log1p so
// they stay finite as two singular values coincide. The diagonal and parameter derivatives come
// from a hand-written reverse sweep through the principal-space chain, including the implicit
// overstress solve (derivatives as in the reference's SolveOverstressGradient, ding.py:90-100).
// In gas mode the end-state porosity of the coupled solve (porous_return.py:43-61) is reversed
// through its converged consistency equation, and the volume rescaling of Fe (ding.py:200-205)
// as a common factor of its principal values.
// Differentiable parameters: shear modulus, Lame lambda, the viscosity parameter and the
// per-particle temperature (through the yield and viscosity factor tables). The gelation latch and
// the wall and stencil switches are discrete; like the reference, no gradient flows through them.
#include <climits>
#include <cstdio>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"

using namespace bk;

namespace {

constexpr int kThreads = 128;

struct AdjParams {
    int64_t n, pitch;
    int R, bc;
    float origin[3], dx, dt, gravity[3];
    int material;  // 0 neo-Hookean, 1 Ding
    int transport; // temperature is a transport field: its adjoint here is that of this substep's T_mat
    DingParamsDev ding;
};

// The loaf and dough configuration (Ding with temperature-dependent parameters, thermal-water
// transport): kernel instances for it take these flags as compile-time constants.
__device__ __forceinline__ void fix_loaf_mode(AdjParams& P) {
    P.material = 1;
    P.transport = 1;
    P.ding.temperature_enabled = 1;
}
bool adj_loaf_mode(const BkSubstepParams& p) {
    return p.material == 1 && p.transport && p.ding.temperature_enabled;
}

// Adjoint of a particle state: same planes as BkState.
struct AdjState {
    float *x, *v, *C, *F, *Fe, *tau, *porosity, *temperature, *mass;
};

// Slots of the principal-space derivative vector: the three singular values, then the parameters.
enum { kS0 = 0, kS1, kS2, kMu, kLam, kTy, kEta, kA, kDirs };

// Forward values of sigma -> (g, h) of the Ding return map (ding.py:103-131), kept for the
// reverse sweep: Fe' = U diag(g) V^T, tau' = U diag(h = cs) U^T.
struct PrincipalFwd {
    float s[3], eps[3], ts[3], dev[3], cs[3], gpre[3], g[3];
    float tr, mean, ty, ty2, q2, p2, bulk, d, h, r, u, w, cm, c;
    float mu, lam, eta, a, dt;
    bool yielded, iso;
};

__device__ PrincipalFwd principal_forward(const float* s, const float* e, float mu, float lam, float ty, float eta, float a,
                                          float dt) {
    PrincipalFwd f;
    f.mu = mu; f.lam = lam; f.ty = ty; f.eta = eta; f.a = a; f.dt = dt;
#pragma unroll
    for (int k = 0; k < 3; ++k) { f.s[k] = s[k]; f.eps[k] = e[k]; }
    f.tr = f.eps[0] + f.eps[1] + f.eps[2];
#pragma unroll
    for (int k = 0; k < 3; ++k) f.ts[k] = 2.f * mu * f.eps[k] + lam * f.tr;
    f.mean = (f.ts[0] + f.ts[1] + f.ts[2]) / 3.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) f.dev[k] = f.ts[k] - f.mean;
    f.ty2 = ty * ty;
    f.q2 = 1.5f * (f.dev[0] * f.dev[0] + f.dev[1] * f.dev[1] + f.dev[2] * f.dev[2]) / f.ty2;
    f.p2 = a * f.mean * f.mean / f.ty2;
    f.bulk = 2.f * mu + 3.f * lam;
    f.d = 6.f * mu * dt * f.ty2 / eta;
    f.h = 2.f / 3.f * dt * a * f.bulk * f.ty2 / eta;
    f.r = solve_overstress(f.q2, f.p2, f.d, f.h);
    f.yielded = f.q2 + f.p2 > 1.0f;
    f.u = 1.f + f.d * f.r;
    f.w = 1.f + f.h * f.r;
#pragma unroll
    for (int k = 0; k < 3; ++k) f.cs[k] = f.dev[k] / f.u + f.mean / f.w;
    f.cm = (f.cs[0] + f.cs[1] + f.cs[2]) / 3.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) f.gpre[k] = expf((f.cs[k] - f.cm) / (2.f * mu) + f.cm / f.bulk);
    f.iso = a == 0.0f;
    f.c = 1.f;
    if (f.iso) {
        // Isochoric correction (ding.py:129-131): Fe' *= cbrt(det trial / det Fe'), a common factor.
        f.c = cbrtf((s[0] * s[1] * s[2]) / (f.gpre[0] * f.gpre[1] * f.gpre[2]));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) f.g[k] = f.gpre[k] * f.c;
    return f;
}

// Reverse sweep of principal_forward: given dL/dg (gb) and dL/dh (hb), the derivatives of L with
// respect to the slots kS0..kA. The overstress root enters through the implicit function theorem
// on R(r) = r + 1 - q2/(1+dr)^2 - p2/(1+hr)^2 (the derivatives of the reference's
// SolveOverstressGradient, ding.py:90-100).
__device__ void principal_vjp(const PrincipalFwd& f, const float* gb, const float* hb, float* out) {
    const float mu = f.mu, lam = f.lam;
    float sb[3] = {0.f, 0.f, 0.f}, gpb[3];
    float mub = 0.f, lamb = 0.f, etab = 0.f, ab = 0.f, ty2b = 0.f;
    if (f.iso) {
        float cb = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            cb += gb[k] * f.gpre[k];
            gpb[k] = gb[k] * f.c;
        }
        // c = cbrt(P), P = s0 s1 s2 / (gp0 gp1 gp2): dc/dP P = c / 3
        const float cp = cb * f.c / 3.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            sb[k] += cp / f.s[k];
            gpb[k] -= cp / f.gpre[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) gpb[k] = gb[k];
    }
    // gpre_k = exp(z_k), z_k = (cs_k - cm) / (2 mu) + cm / bulk
    float csb[3], cmb = 0.f, bulkb = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float zb = gpb[k] * f.gpre[k];
        csb[k] = hb[k] + zb / (2.f * mu);
        cmb += zb * (1.f / f.bulk - 1.f / (2.f * mu));
        mub -= zb * (f.cs[k] - f.cm) / (2.f * mu * mu);
        bulkb -= zb * f.cm / (f.bulk * f.bulk);
    }
    // cm = (cs_0 + cs_1 + cs_2) / 3; cs_k = dev_k / u + mean / w
    float devb[3], meanb = 0.f, ub = 0.f, wb = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        csb[k] += cmb / 3.f;
        devb[k] = csb[k] / f.u;
        meanb += csb[k] / f.w;
        ub -= csb[k] * f.dev[k] / (f.u * f.u);
        wb -= csb[k] * f.mean / (f.w * f.w);
    }
    float db = ub * f.r, hbar = wb * f.r;
    const float rb = ub * f.d + wb * f.h;
    float q2b = 0.f, p2b = 0.f;
    if (f.yielded) {
        const float u3 = f.u * f.u * f.u, w3 = f.w * f.w * f.w;
        const float Rr = 1.f + 2.f * f.d * f.q2 / u3 + 2.f * f.h * f.p2 / w3;
        const float k = -rb / Rr;
        q2b += k * (-1.f / (f.u * f.u));
        p2b += k * (-1.f / (f.w * f.w));
        db += k * (2.f * f.q2 * f.r / u3);
        hbar += k * (2.f * f.p2 * f.r / w3);
    }
    // h = (2/3) dt a bulk ty2 / eta
    const float kh = 2.f / 3.f * f.dt / f.eta;
    ab += hbar * kh * f.bulk * f.ty2;
    bulkb += hbar * kh * f.a * f.ty2;
    ty2b += hbar * kh * f.a * f.bulk;
    etab -= hbar * f.h / f.eta;
    // d = 6 mu dt ty2 / eta
    mub += db * 6.f * f.dt * f.ty2 / f.eta;
    ty2b += db * 6.f * mu * f.dt / f.eta;
    etab -= db * f.d / f.eta;
    // bulk = 2 mu + 3 lam
    mub += 2.f * bulkb;
    lamb += 3.f * bulkb;
    // p2 = a mean^2 / ty2; q2 = 1.5 |dev|^2 / ty2
    ab += p2b * f.mean * f.mean / f.ty2;
    meanb += p2b * 2.f * f.a * f.mean / f.ty2;
    ty2b -= p2b * f.p2 / f.ty2;
#pragma unroll
    for (int k = 0; k < 3; ++k) devb[k] += q2b * 3.f * f.dev[k] / f.ty2;
    ty2b -= q2b * f.q2 / f.ty2;
    const float tyb = 2.f * f.ty * ty2b;
    // dev_k = ts_k - mean; mean = (ts_0 + ts_1 + ts_2) / 3
    float tsb[3], devsum = devb[0] + devb[1] + devb[2];
    meanb -= devsum;
#pragma unroll
    for (int k = 0; k < 3; ++k) tsb[k] = devb[k] + meanb / 3.f;
    // ts_k = 2 mu eps_k + lam tr; tr = eps_0 + eps_1 + eps_2; eps_k = log s_k
    const float tsum = tsb[0] + tsb[1] + tsb[2];
    lamb += f.tr * tsum;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        mub += 2.f * f.eps[k] * tsb[k];
        sb[k] += (2.f * mu * tsb[k] + lam * tsum) / f.s[k];
    }
    out[kS0] = sb[0]; out[kS1] = sb[1]; out[kS2] = sb[2];
    out[kMu] = mub; out[kLam] = lamb; out[kTy] = tyb; out[kEta] = etab; out[kA] = ab;
}

// Inputs of the end-state porosity solve of gas mode (ding.py:183-196), computed from the trial
// singular values in the forward's order of operations.
struct CoupledFwd {
    float eps[3], dev[3], tr, mean, ty, ty2, q, p, df, ms, ex, bulk, mu, lam, eta, dt;
    double Vp;
};

__device__ CoupledFwd coupled_forward(const float* e, float mu, float lam, float ty, float eta, float dt, float n0,
                                      float por) {
    CoupledFwd c;
    c.mu = mu; c.lam = lam; c.ty = ty; c.eta = eta; c.dt = dt;
#pragma unroll
    for (int k = 0; k < 3; ++k) c.eps[k] = e[k];
    c.tr = c.eps[0] + c.eps[1] + c.eps[2];
    float ts[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ts[k] = 2.0f * mu * c.eps[k] + lam * c.tr;
    c.mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) c.dev[k] = ts[k] - c.mean;
    c.ty2 = ty * ty;
    c.q = 1.5f * (c.dev[0] * c.dev[0] + c.dev[1] * c.dev[1] + c.dev[2] * c.dev[2]) / c.ty2;
    c.p = c.mean * c.mean / c.ty2;
    c.df = 6.0f * mu * dt * ty * ty / eta;
    c.bulk = 2.0f * mu + 3.0f * lam;
    c.ms = 2.0f / 3.0f * c.bulk * dt * ty * ty / eta;
    c.ex = 3.0f * c.mean / c.bulk;
    c.Vp = 1.0 - (double)n0 + (double)por;
    return c;
}

// End-state porosity of gas mode, n = solve_porosity(q, p, d, h, e, Vp) for the trial singular
// values s (ding.py:183-197), and its gradient G = dn/d(s0, s1, s2, mu, lambda, yield stress,
// viscosity, old porosity). n is the root of n = pred(n; q, p, d, h, e, Vp) with
// pred = Vp exp(e (1 - 1/v)) - 1 + n0, v = 1 + h a(n) r and r the overstress root of
// r + 1 - q/(1+dr)^2 - a p/(1+h a r)^2 = 0; the implicit function theorem on the converged
// equation (the derivatives of the reference's SolvePorosityGradient, porous_return.py:64-100)
// gives dn/dtheta = dpred/dtheta / (1 - dpred/dn); the elastic early exit is the case r = 0.
// Out of line, called before the rest of the reverse sweep needs its registers.
__device__ __noinline__ float coupled_solve_grad(const float* s, const float* log_s, float mu, float lam, float ty, float eta, float dt,
                                                 float n0, float por, float* G) {
    const CoupledFwd c = coupled_forward(log_s, mu, lam, ty, eta, dt, n0, por);
    double r = 0.0;
    bool elastic_exit;
    const float nf = solve_porosity(c.q, c.p, c.df, c.ms, c.ex, c.Vp, n0, &r, &elastic_exit);
    if (elastic_exit) {
        // Certain elastic exit: q + a(nf) p <= 1, so r = 0, v = 1, E = 1 and every derivative below
        // is an exact zero except dn/dVp = 1 (the same values the general path computes for finite
        // parameters).
#pragma unroll
        for (int k = 0; k < 7; ++k) G[k] = 0.f;
        G[7] = 1.f;
        return nf;
    }
    const double n = (double)nf;
    const double q = c.q, p = c.p, d = c.df, h = c.ms, e = c.ex, Vp = c.Vp;
    const double a = pressure_coefficient64(n);
    r = overstress64(q, a * p, d, h * a, &r);
    const double v = 1.0 + h * a * r;
    const double E = exp(e * (1.0 - 1.0 / v));
    const double K = Vp * E * e / (v * v);  // dpred/dv
    double da = 0.0;
    if (n > 0.0) {
        const double lg = log(1.0 / n);
        da = a * (2.0 / (n * lg) - 3.5 / (3.5 * n + 1.0));
    }
    double rq = 0.0, rp = 0.0, rd = 0.0, rh = 0.0;  // dr/d(q, a p, d, h a)
    if (q + a * p > 1.0) {
        const double u = 1.0 + d * r;
        const double Fr = 1.0 + 2.0 * d * q / (u * u * u) + 2.0 * h * a * a * p / (v * v * v);
        rq = 1.0 / (u * u * Fr);
        rp = 1.0 / (v * v * Fr);
        rd = -2.0 * q * r / (u * u * u * Fr);
        rh = -2.0 * a * p * r / (v * v * v * Fr);
    }
    const double slope = K * h * da * (r + a * (rp * p + rh * h));
    const double lm = 1.0 / (1.0 - slope);
    const float qb = (float)(lm * K * h * a * rq);
    const float pb = (float)(lm * K * h * a * a * rp);
    const float db = (float)(lm * K * h * a * rd);
    const float hb = (float)(lm * K * (a * r + h * a * a * rh));
    const float eb = (float)(lm * Vp * E * (1.0 - 1.0 / v));
    // q = 1.5 |dev|^2 / ty2, p = mean^2 / ty2, d = 6 mu dt ty2 / eta, h = (2/3) bulk dt ty2 / eta,
    // e = 3 mean / bulk
    float devb[3], meanb = 0.f, ty2b = 0.f, mub = 0.f, lamb = 0.f, etab = 0.f, bulkb = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) devb[k] = qb * 3.f * c.dev[k] / c.ty2;
    ty2b -= qb * c.q / c.ty2;
    meanb += pb * 2.f * c.mean / c.ty2;
    ty2b -= pb * c.p / c.ty2;
    mub += db * 6.f * c.dt * c.ty2 / c.eta;
    ty2b += db * 6.f * c.mu * c.dt / c.eta;
    etab -= db * c.df / c.eta;
    bulkb += hb * (2.f / 3.f) * c.dt * c.ty2 / c.eta;
    ty2b += hb * (2.f / 3.f) * c.bulk * c.dt / c.eta;
    etab -= hb * c.ms / c.eta;
    meanb += eb * 3.f / c.bulk;
    bulkb -= eb * c.ex / c.bulk;
    mub += 2.f * bulkb;
    lamb += 3.f * bulkb;
    // dev_k = ts_k - mean, mean = sum ts / 3, ts_k = 2 mu eps_k + lam tr, eps_k = log s_k
    meanb -= devb[0] + devb[1] + devb[2];
    float tsb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) tsb[k] = devb[k] + meanb / 3.f;
    const float tsum = tsb[0] + tsb[1] + tsb[2];
    lamb += c.tr * tsum;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        mub += 2.f * c.eps[k] * tsb[k];
        G[k] = (2.f * c.mu * tsb[k] + c.lam * tsum) / s[k];
    }
    G[3] = mub;
    G[4] = lamb;
    G[5] = 2.f * c.ty * ty2b;
    G[6] = etab;
    G[7] = (float)(lm * E);  // through Vp = 1 - n0 + n_old
    return nf;
}

__device__ __forceinline__ void add_m3(float* __restrict__ p, int64_t i, int64_t pitch, const float* a) {
#pragma unroll
    for (int c = 0; c < 9; ++c) p[c * pitch + i] += a[c];
}

// a^T b and a b^T for 3x3 row-major matrices.
__device__ __forceinline__ M3 mul_tn(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[3 * i + j] = a.m[i] * b.m[j] + a.m[3 + i] * b.m[3 + j] + a.m[6 + i] * b.m[6 + j];
    return r;
}
__device__ __forceinline__ M3 mul_nt(const M3& a, const M3& b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            r.m[3 * i + j] = a.m[3 * i] * b.m[3 * j] + a.m[3 * i + 1] * b.m[3 * j + 1] + a.m[3 * i + 2] * b.m[3 * j + 2];
    return r;
}

// Block-reduce a value into one float64 accumulator (material parameter adjoints).
__device__ void block_accumulate(double* target, float value) {
    __shared__ float s_part[kThreads / 32];
    float v = value;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < kThreads / 32; ++w) t += s_part[w];
        if (t != 0.f) atomicAdd(target, (double)t);
    }
    __syncthreads();
}

// Quadratic B-spline weight derivative dN_o(l)/dl (transfer.py:4-13).
__device__ __forceinline__ float qweight_grad(float l, int o) {
    if (o == 0) return -(1.5f - l);
    if (o == 1) return -2.f * (l - 1.f);
    return l - 0.5f;
}

// ------------------------------------------------------------ G2P + return
// params_adj: float64 [0] mu, [1] lambda, [2] viscosity parameter.
// kCoupled: gas mode's coupled porosity (a separate instance, so the other modes keep their registers).
// kLoaf: the loaf configuration (Ding with temperature, transport) as compile-time constants.
template <bool kCoupled, bool kLoaf = false>
__global__ void __launch_bounds__(kThreads, 4) k_adj_g2p_return(AdjParams P, BkState in, const float4* __restrict__ grid_v,
                                                          const float* __restrict__ eta_param, AdjState out_adj,
                                                          AdjState in_adj, double* __restrict__ params_adj) {
    if constexpr (kLoaf) fix_loaf_mode(P);
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    float acc_mu = 0.f, acc_lam = 0.f, acc_eta = 0.f;
    if (i < P.n) {
        const int64_t pitch = P.pitch;
        V3 xi = load_v3(in.x, i, pitch);
        Stencil st = make_stencil(xi, P.origin, P.dx, P.R);
        if (st.valid) {
            // ---- forward recompute: G2P (C' only; v' does not enter the reverse sweep)
            float nc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            const float k4 = 4.0f / (P.dx * P.dx);
#pragma unroll
            for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                    for (int oz = 0; oz < 3; ++oz) {
                        float w = st.w[0][ox] * st.w[1][oy] * st.w[2][oz];
                        float d[3] = {((float)ox - st.l[0]) * P.dx, ((float)oy - st.l[1]) * P.dx, ((float)oz - st.l[2]) * P.dx};
                        float4 u = __ldg(grid_v + node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R));
                        float uu[3] = {u.x, u.y, u.z};
#pragma unroll
                        for (int r = 0; r < 3; ++r)
#pragma unroll
                            for (int c = 0; c < 3; ++c) nc[3 * r + c] += k4 * w * (uu[r] * d[c]);
                    }
            M3 F = load_m3(in.F, i, pitch);
            M3 G;
#pragma unroll
            for (int e = 0; e < 9; ++e) G.m[e] = P.dt * nc[e] + ((e % 4) == 0 ? 1.f : 0.f);
            M3 Fn = matmul(G, F);
            // ---- adjoints of the substep's outputs
            float xb[3], vb[3], Cb[9], Fb[9];
#pragma unroll
            for (int c = 0; c < 3; ++c) { xb[c] = out_adj.x[c * pitch + i]; vb[c] = out_adj.v[c * pitch + i]; }
#pragma unroll
            for (int c = 0; c < 9; ++c) { Cb[c] = out_adj.C[c * pitch + i]; Fb[c] = out_adj.F[c * pitch + i]; }
            float Tb = 0.f;
            float Feb_in[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            float porb_in = 0.f;
            if (P.material == 1) {
                const DingParamsDev& D = P.ding;
                float Fe_b[9], tau_b[9];
#pragma unroll
                for (int c = 0; c < 9; ++c) { Fe_b[c] = out_adj.Fe[c * pitch + i]; tau_b[c] = out_adj.tau[c * pitch + i]; }
                float por_b = out_adj.porosity[i];
                Tb = P.transport ? 0.f : out_adj.temperature[i];
                float por = in.porosity[i];
                int gel = in.gelled[i];
                float T = in.material_temperature[i];
                // temperature tables (ding.py:159-171)
                float Teff = T, ty = D.yield_stress, eta = __ldg(eta_param);
                float dty_dT = 0.f, deta_dT = 0.f, eta_factor = 1.f;
                if (D.temperature_enabled) {
                    if (T >= D.knots[3]) gel = 1;
                    if (gel) Teff = D.knots[3];
                    float fy = temperature_factor(Teff, D.knots, D.yield_factors);
                    float fv = temperature_factor(Teff, D.knots, D.viscosity_factors);
                    ty = D.yield_stress * fy;
                    eta_factor = fv;
                    eta = eta * fv;
                    if (!gel) {
                        // slope of the piecewise-linear tables at T (zero outside the knots)
                        for (int k = 0; k < 3; ++k) {
                            if (T >= D.knots[k] && T < D.knots[k + 1]) {
                                float span = D.knots[k + 1] - D.knots[k];
                                dty_dT = D.yield_stress * (D.yield_factors[k + 1] - D.yield_factors[k]) / span;
                                deta_dT = __ldg(eta_param) * (D.viscosity_factors[k + 1] - D.viscosity_factors[k]) / span;
                            }
                        }
                    }
                }
                M3 Fe_old = load_m3(in.Fe, i, pitch);
                M3 Gd;
#pragma unroll
                for (int e = 0; e < 9; ++e) Gd.m[e] = D.dt * nc[e] + ((e % 4) == 0 ? 1.f : 0.f);
                M3 trial = matmul(Gd, Fe_old);
                M3 U, V;
                float s[3], se[3];
                svd3f(trial, U, s, V, se);
                // Gas mode: the end-state porosity n_ret of the coupled solve sets a(n) of the
                // return, and the returned Fe is rescaled to det F' / (1 - n0 + n_ret) (ding.py:183-205).
                constexpr bool coupled = kCoupled;
                float n_ret = por;
                float nG[8];  // dn_ret/d(s0, s1, s2, mu, lambda, yield, viscosity, old porosity)
                if (coupled) n_ret = coupled_solve_grad(s, se, D.mu, D.lam, ty, eta, D.dt, D.initial_porosity, por, nG);
                float a = porosity_coefficient(n_ret);
                PrincipalFwd pr = principal_forward(s, se, D.mu, D.lam, ty, eta, a, D.dt);
                bool porosity_free = !(D.initial_porosity == 0.0f && por == 0.0f);
                float detFn = det3(Fn);
                float gv[3] = {pr.g[0], pr.g[1], pr.g[2]};  // principal values of the stored Fe'
                float gb_por[3] = {0.f, 0.f, 0.f};
                double nret_b = 0.0;
                float cg = 1.f, target = 1.f;
                if (coupled) {
                    target = (float)(1.0 - (double)D.initial_porosity + (double)n_ret);
                    cg = cbrt_near_one((double)detFn / ((double)target * ((double)pr.g[0] * pr.g[1] * pr.g[2])));
#pragma unroll
                    for (int k = 0; k < 3; ++k) gv[k] *= cg;
                    if (porosity_free) nret_b += por_b;  // porosity' = n_ret
                } else if (porosity_free && por_b != 0.f) {
                    // porosity' = det(F') / prod(g) - 1 + n0 (uncoupled; zero when n0 = n = 0)
                    float npor = detFn / (pr.g[0] * pr.g[1] * pr.g[2]);
                    // d/dF' det(F') = det(F') F'^-T
                    M3 inv = inverse3(Fn);
                    float scale_f = por_b * npor;
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int c = 0; c < 3; ++c) Fb[3 * r + c] += scale_f * inv.m[3 * c + r];
#pragma unroll
                    for (int k = 0; k < 3; ++k) gb_por[k] = -por_b * npor / pr.g[k];
                }
                // rotated adjoints Gh = U^T Fe_bar V, Th = U^T tau_bar U
                M3 FeB, tauB;
#pragma unroll
                for (int e = 0; e < 9; ++e) { FeB.m[e] = Fe_b[e]; tauB.m[e] = tau_b[e]; }
                const M3 Ghm = mul_tn(U, matmul(FeB, V)), Thm = mul_tn(U, matmul(tauB, U));
                const float* Gh = Ghm.m;
                const float* Th = Thm.m;
                // diagonal: sbar_j = sum_i (Gh_ii + gb_por_i) dg_i/ds_j + Th_ii dh_i/ds_j; parameters likewise
                M3 Abm;
                float* Ab = Abm.m;
                float dpar[kDirs];
                {
                    float gbar[3] = {Gh[0] + gb_por[0], Gh[4] + gb_por[1], Gh[8] + gb_por[2]};
                    if (coupled) {
                        // g'_k = cg g_k, cg = cbrt(det F' / (target prod g)): a common factor
                        const float cgb = (Gh[0] * pr.g[0] + Gh[4] * pr.g[1] + Gh[8] * pr.g[2]) * (1.f / 3.f);
#pragma unroll
                        for (int k = 0; k < 3; ++k) gbar[k] = cg * (gbar[k] - cgb / pr.g[k]);
                        const float lb = cgb * cg;  // dL/d log(det F' / target)
                        M3 inv = inverse3(Fn);
#pragma unroll
                        for (int r = 0; r < 3; ++r)
#pragma unroll
                            for (int c = 0; c < 3; ++c) Fb[3 * r + c] += lb * inv.m[3 * c + r];
                        nret_b -= (double)(lb / target);
                    }
                    const float hbar[3] = {Th[0], Th[4], Th[8]};
                    principal_vjp(pr, gbar, hbar, dpar);
                }
                float porb_coupled = 0.f;
                if (coupled) {
                    // a = a(n_ret), then the solve's inputs (s, mu, lambda, yield, viscosity, old n)
                    if (n_ret > 0.0f) {
                        const float lg = logf(1.0f / n_ret);
                        nret_b += (double)(dpar[kA] * a * (2.0f / (n_ret * lg) - 3.5f / (3.5f * n_ret + 1.0f)));
                    }
                    const float nb = (float)nret_b;
#pragma unroll
                    for (int k = 0; k < 3; ++k) dpar[kS0 + k] += nb * nG[k];
                    dpar[kMu] += nb * nG[3];
                    dpar[kLam] += nb * nG[4];
                    dpar[kTy] += nb * nG[5];
                    dpar[kEta] += nb * nG[6];
                    porb_coupled = nb * nG[7];
                }
                Ab[0] = dpar[kS0];
                Ab[4] = dpar[kS1];
                Ab[8] = dpar[kS2];
                // Off-diagonal terms, one unordered pair (p, q) at a time. With M = U^T dA V:
                //   dFe^_pq = P_pq M_pq + Q_pq M_qp, P_pq = (g_q s_q - g_p s_p) / (s_q^2 - s_p^2),
                //   Q_pq = (g_q s_p - g_p s_q) / (s_q^2 - s_p^2); dtau^_pq = D (s_q M_pq + s_p M_qp),
                //   D = (h_q - h_p) / (s_q^2 - s_p^2), symmetric in (p, q).
                // With L = log(s_q / s_p): s_q = s_p (1 + A), g_q = g_p (1 + B), A = expm1(L),
                // B = expm1(L / (1 + d r)), so the divided difference (g_q - g_p) / (s_q - s_p) is
                // (g_p / s_p) B / A and h_q - h_p = 2 mu L / (1 + d r): one log1p and two expm1 per pair,
                // finite as the two singular values coincide.
                const float one_dr = 1.f + pr.d * pr.r;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const int p = k == 2 ? 1 : 0;
                    const int q = k == 0 ? 1 : 2;
                    const float sp = s[p], sq = s[q], gp = gv[p], gq = gv[q];
                    const float L = log1pf((sq - sp) / sp);
                    float ratio = 1.f / one_dr, xo = 1.f;
                    if (fabsf(L) >= 1e-12f) {
                        const float A = expm1f(L), B = expm1f(L / one_dr);
                        ratio = B / A;
                        xo = L / A;
                    }
                    const float ddg = (gp / sp) * ratio;
                    const float inv_sum = 1.f / (sp + sq);
                    const float P_pq = (ddg * sq + gp) * inv_sum, Q_qp = (ddg * sq - gq) * inv_sum;
                    const float P_qp = (ddg * sp + gq) * inv_sum, Q_pq = (ddg * sp - gp) * inv_sum;
                    const float Dm = 2.f * D.mu * xo * inv_sum / (one_dr * sp);
                    const float Tsym = Th[3 * p + q] + Th[3 * q + p];
                    Ab[3 * p + q] = Gh[3 * p + q] * P_pq + Gh[3 * q + p] * Q_qp + Tsym * Dm * sq;
                    Ab[3 * q + p] = Gh[3 * q + p] * P_qp + Gh[3 * p + q] * Q_pq + Tsym * Dm * sp;
                }
                // trial adjoint A_bar = U Ab V^T
                const M3 Tbm = matmul(U, mul_nt(Abm, V));
                const float* Tb_m = Tbm.m;
                // trial = (I + dt C') Fe: Cbar += dt trial_bar Fe^T; Fe_bar_in = (I + dt C')^T trial_bar
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float tc = 0.f, fe = 0.f;
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            tc += Tb_m[3 * r + k] * Fe_old.m[3 * c + k];
                            fe += Gd.m[3 * k + r] * Tb_m[3 * k + c];
                        }
                        Cb[3 * r + c] += D.dt * tc;
                        Feb_in[3 * r + c] = fe;
                    }
                // parameters: eta = eta_param * fv(T); ty = ys * fy(T)
                acc_mu = dpar[kMu];
                acc_lam = dpar[kLam];
                acc_eta = dpar[kEta] * eta_factor;
                Tb += dpar[kTy] * dty_dT + dpar[kEta] * deta_dT;
                // porosity -> a(n) (zero at n = 0); in gas mode through the coupled solve
                if (coupled) {
                    porb_in = porb_coupled;
                } else if (por > 0.0f) {
                    float lg = logf(1.0f / por);
                    float da = a * (2.0f / (por * lg) - 3.5f / (3.5f * por + 1.0f));
                    porb_in = dpar[kA] * da;
                }
            }
            // ---- G2P backward, per particle: x' = x + dt v'; F' = (I + dt C') F. The node scatter
            // of v-bar and C-bar and the weight gradients of x follow in k_adj_g2p_scatter, which
            // takes v-bar and C-bar from in_adj.v and in_adj.C (k_adj_p2g overwrites both later).
#pragma unroll
            for (int r = 0; r < 3; ++r) vb[r] += P.dt * xb[r];
            float Fb_in[9];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float fc = 0.f, cc = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        fc += G.m[3 * k + r] * Fb[3 * k + c];
                        cc += Fb[3 * r + k] * F.m[3 * c + k];
                    }
                    Fb_in[3 * r + c] = fc;
                    Cb[3 * r + c] += P.dt * cc;
                }
#pragma unroll
            for (int c = 0; c < 3; ++c) in_adj.v[c * pitch + i] = vb[c];
#pragma unroll
            for (int e = 0; e < 9; ++e) in_adj.C[e * pitch + i] = Cb[e];
            // F (of state t): from G2P; C gets no direct dependence from G2P (C' does)
            M3 fbm;
#pragma unroll
            for (int e = 0; e < 9; ++e) fbm.m[e] = Fb_in[e];
            store_m3(in_adj.F, i, pitch, fbm);
            if (P.material == 1) {
                M3 feb;
#pragma unroll
                for (int e = 0; e < 9; ++e) feb.m[e] = Feb_in[e];
                store_m3(in_adj.Fe, i, pitch, feb);
                in_adj.porosity[i] = porb_in;
                in_adj.temperature[i] = Tb;
            }
        } else {
            // The forward raised the stencil flag for this particle; its adjoint is zero (x: in
            // k_adj_g2p_scatter).
#pragma unroll
            for (int c = 0; c < 9; ++c) in_adj.F[c * pitch + i] = 0.f;
            if (P.material == 1) {
#pragma unroll
                for (int c = 0; c < 9; ++c) in_adj.Fe[c * pitch + i] = 0.f;
                in_adj.porosity[i] = 0.f;
                in_adj.temperature[i] = P.transport ? 0.f : out_adj.temperature[i];
            }
        }
    }
    if (params_adj) {
        block_accumulate(params_adj + 0, acc_mu);
        block_accumulate(params_adj + 1, acc_lam);
        block_accumulate(params_adj + 2, acc_eta);
    }
}

// ------------------------------------------------------------ G2P scatter
// The node-velocity adjoint of G2P (transfer.py:90-104 reversed): node j receives
// w_j (v-bar + 4/dx^2 C-bar d_j) with d_j = (o_j - l) dx, i.e. w_j (q + A o_j) with
// q = v-bar - (4/dx) C-bar l and A = (4/dx) C-bar -- the forward P2G's form, scattered the same
// way: runs of particles with one stencil base within a warp, lane j < 27 summing node j over the
// run, a shared-memory tile over the block's node box (when it fits kTileNodes) and one global
// atomic per tile node. Each particle also gathers the weight gradients of x (reads only).
constexpr int kTileNodes = 512;

// A particle's record: stencil weights as padded axis rows (a lane reads row 3a + o of its node
// offsets without selects), and {q0 q1 q2 A0} {A1 A2 A3 A4} {A5 A6 A7 A8} as 128-bit broadcasts.
struct ScatterSmem {
    float4 val[kThreads][3];
    float w[9][kThreads + 1];
    float4 tile[kTileNodes];
    int box[6];
};

template <bool kLoaf = false>
__global__ void __launch_bounds__(kThreads) k_adj_g2p_scatter(AdjParams P, BkState in, const float4* __restrict__ grid_v,
                                                            AdjState out_adj, AdjState in_adj,
                                                            float4* __restrict__ grid_v_adj) {
    if constexpr (kLoaf) fix_loaf_mode(P);
    __shared__ ScatterSmem sm;
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t i = blockIdx.x * (int64_t)kThreads + tid;
    const int64_t pitch = P.pitch;
    Stencil st;
    st.valid = false;
    st.b[0] = st.b[1] = st.b[2] = 0;
    if (i < P.n) st = make_stencil(load_v3(in.x, i, pitch), P.origin, P.dx, P.R);
    const bool valid = i < P.n && st.valid;
    float q[3] = {0.f, 0.f, 0.f}, A[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (valid) {
        const float k4 = 4.0f / (P.dx * P.dx), inv_dx = 1.f / P.dx;
        float vb[3], Cb[9], xg[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            vb[c] = in_adj.v[c * pitch + i];
            xg[c] = out_adj.x[c * pitch + i];
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) Cb[e] = in_adj.C[e * pitch + i];
#pragma unroll
        for (int ox = 0; ox < 3; ++ox)
#pragma unroll
            for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) {
                    const int o[3] = {ox, oy, oz};
                    const float wa[3] = {st.w[0][ox], st.w[1][oy], st.w[2][oz]};
                    const float w = wa[0] * wa[1] * wa[2];
                    const float d[3] = {((float)ox - st.l[0]) * P.dx, ((float)oy - st.l[1]) * P.dx,
                                        ((float)oz - st.l[2]) * P.dx};
                    const float4 u = __ldg(grid_v + node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R));
                    const float uu[3] = {u.x, u.y, u.z};
                    // the weight's cofactor s = vb . u + k u^T Cb d
                    float sdot = vb[0] * uu[0] + vb[1] * uu[1] + vb[2] * uu[2];
                    float cu[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) cu[c] = Cb[c] * uu[0] + Cb[3 + c] * uu[1] + Cb[6 + c] * uu[2];
                    sdot += k4 * (cu[0] * d[0] + cu[1] * d[1] + cu[2] * d[2]);
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const float dw = qweight_grad(st.l[a], o[a]) * inv_dx;
                        float rest = 1.f;
#pragma unroll
                        for (int b2 = 0; b2 < 3; ++b2)
                            if (b2 != a) rest *= wa[b2];
                        xg[a] += dw * rest * sdot - k4 * w * cu[a];  // d = x_i - x_p: dd/dx_p = -I
                    }
                }
        store_v3(in_adj.x, i, pitch, V3{{xg[0], xg[1], xg[2]}});
        const float kd = k4 * P.dx;
#pragma unroll
        for (int r = 0; r < 3; ++r)
            q[r] = vb[r] - kd * (Cb[3 * r] * st.l[0] + Cb[3 * r + 1] * st.l[1] + Cb[3 * r + 2] * st.l[2]);
#pragma unroll
        for (int e = 0; e < 9; ++e) A[e] = kd * Cb[e];
    } else if (i < P.n) {
#pragma unroll
        for (int c = 0; c < 3; ++c) in_adj.x[c * pitch + i] = 0.f;
    }
    {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int o = 0; o < 3; ++o) sm.w[3 * a + o][tid] = valid ? st.w[a][o] : 0.f;
        sm.val[tid][0] = make_float4(q[0], q[1], q[2], A[0]);
        sm.val[tid][1] = make_float4(A[1], A[2], A[3], A[4]);
        sm.val[tid][2] = make_float4(A[5], A[6], A[7], A[8]);
    }
    if (tid < 6) sm.box[tid] = tid < 3 ? INT_MAX : INT_MIN;
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int lo = __reduce_min_sync(0xffffffffu, valid ? st.b[a] : INT_MAX);
        const int hi = __reduce_max_sync(0xffffffffu, valid ? st.b[a] + 2 : INT_MIN);
        if (lane == 0 && lo != INT_MAX) {
            atomicMin(&sm.box[a], lo);
            atomicMax(&sm.box[3 + a], hi);
        }
    }
    __syncthreads();
    int lo[3] = {0, 0, 0}, ext[3] = {1, 1, 1};
    int count = 0;
    bool tiled = false;
    if (sm.box[0] != INT_MAX) {
        long long c = 1;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = sm.box[a];
            ext[a] = sm.box[3 + a] - sm.box[a] + 1;
            c *= ext[a];
        }
        tiled = c <= kTileNodes;
        count = tiled ? (int)c : 0;
    }
    for (int t = tid; t < count; t += kThreads) sm.tile[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    const long long key = valid ? (((long long)st.b[0] << 42) | ((long long)st.b[1] << 21) | (long long)st.b[2]) : -1;
    const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
    unsigned starts = __ballot_sync(0xffffffffu, valid && (lane == 0 || prev != key));
    const int warp_base = tid & ~31;
    const int ox = (lane < 27 ? lane : 0) / 9, oy = ((lane < 27 ? lane : 0) / 3) % 3, oz = (lane < 27 ? lane : 0) % 3;
    const float fo[3] = {(float)ox, (float)oy, (float)oz};
    while (starts) {
        const int s0 = __ffs(starts) - 1;
        starts &= starts - 1;
        const int e = starts ? __ffs(starts) - 1 : 32;
        const int b0 = __shfl_sync(0xffffffffu, st.b[0], s0), b1 = __shfl_sync(0xffffffffu, st.b[1], s0),
                  b2 = __shfl_sync(0xffffffffu, st.b[2], s0);
        if (lane < 27) {
            // paired accumulators, one packed multiply-add per pair (ffma2)
            float2 q01 = {0.f, 0.f}, q2A0 = {0.f, 0.f}, A12 = {0.f, 0.f}, A34 = {0.f, 0.f};
            float2 A56 = {0.f, 0.f}, A78 = {0.f, 0.f};
            const float* wx = sm.w[ox];
            const float* wy = sm.w[3 + oy];
            const float* wz = sm.w[6 + oz];
#pragma unroll 2
            for (int k = warp_base + s0; k < warp_base + e; ++k) {
                const float w = wx[k] * wy[k] * wz[k];
                const float2 ww = make_float2(w, w);
                const float4 v0 = sm.val[k][0], v1 = sm.val[k][1], v2 = sm.val[k][2];
                q01 = ffma2(ww, make_float2(v0.x, v0.y), q01);
                q2A0 = ffma2(ww, make_float2(v0.z, v0.w), q2A0);
                A12 = ffma2(ww, make_float2(v1.x, v1.y), A12);
                A34 = ffma2(ww, make_float2(v1.z, v1.w), A34);
                A56 = ffma2(ww, make_float2(v2.x, v2.y), A56);
                A78 = ffma2(ww, make_float2(v2.z, v2.w), A78);
            }
            const float aq[3] = {q01.x, q01.y, q2A0.x};
            const float aA[9] = {q2A0.y, A12.x, A12.y, A34.x, A34.y, A56.x, A56.y, A78.x, A78.y};
            float ap[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) ap[r] = aq[r] + (aA[3 * r] * fo[0] + aA[3 * r + 1] * fo[1] + aA[3 * r + 2] * fo[2]);
            if (tiled) {
                float* cell = reinterpret_cast<float*>(
                    &sm.tile[((b0 + ox - lo[0]) * ext[1] + (b1 + oy - lo[1])) * ext[2] + (b2 + oz - lo[2])]);
                atomicAdd(cell + 0, ap[0]);
                atomicAdd(cell + 1, ap[1]);
                atomicAdd(cell + 2, ap[2]);
            } else {
                atomicAdd(grid_v_adj + node_index(b0 + ox, b1 + oy, b2 + oz, P.R), make_float4(ap[0], ap[1], ap[2], 0.f));
            }
        }
    }
    __syncthreads();
    for (int t = tid; t < count; t += kThreads) {
        const float4 v = sm.tile[t];
        if (v.x == 0.f && v.y == 0.f && v.z == 0.f) continue;
        const int z = t % ext[2], y = (t / ext[2]) % ext[1], x = t / (ext[2] * ext[1]);
        atomicAdd(grid_v_adj + node_index(lo[0] + x, lo[1] + y, lo[2] + z, P.R), v);
    }
}

// ------------------------------------------------------------- grid update
__device__ __forceinline__ void adj_grid_node(const AdjParams& P, const float4* __restrict__ pm,
                                              float4* __restrict__ grid_v_adj, float4* __restrict__ pm_adj,
                                              int64_t i, int c0, int c1, int c2, bool clear) {
    float4 a = grid_v_adj[i];
    float4 q = pm[i];
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    if (q.w > 0.0f && (a.x != 0.f || a.y != 0.f || a.z != 0.f)) {
        const int R = P.R, bc = P.bc;
        const int c[3] = {c0, c1, c2};
        float p[3] = {q.x, q.y, q.z}, ab[3] = {a.x, a.y, a.z};
        float pb[3], mb = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float vel = p[k] / q.w + P.dt * P.gravity[k];
            bool clamped = (c[k] < bc && vel < 0.0f) || (c[k] >= R - bc && vel > 0.0f);
            float g = clamped ? 0.f : ab[k];
            pb[k] = g / q.w;
            mb -= g * p[k] / (q.w * q.w);
        }
        out = make_float4(pb[0], pb[1], pb[2], mb);
    }
    pm_adj[i] = out;
    if (clear) grid_v_adj[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Every node of the grid (velocity adjoint zeroed beforehand by the caller of the substep).
__global__ void k_adj_grid(AdjParams P, const float4* __restrict__ pm, float4* __restrict__ grid_v_adj,
                           float4* __restrict__ pm_adj, int64_t nodes) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const int R = P.R;
    adj_grid_node(P, pm, grid_v_adj, pm_adj, i, (int)(i / ((int64_t)R * R)), (int)((i / R) % R), (int)(i % R), false);
}

// The nodes of the forward substep's active box (inclusive lo[3], hi[3] on the device), which holds
// every stencil node; the velocity adjoint is zeroed behind, so the next call finds it zero.
__global__ void k_adj_grid_box(AdjParams P, const int32_t* __restrict__ box, const float4* __restrict__ pm,
                               float4* __restrict__ grid_v_adj, float4* __restrict__ pm_adj) {
    int lo[3], ext[3];
    int64_t count = 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int l = max(box[a], 0), h = min(box[3 + a], P.R - 1);
        if (l > h) return;
        lo[a] = l;
        ext[a] = h - l + 1;
        count *= ext[a];
    }
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int c2 = lo[2] + (int)(t % ext[2]);
        const int c1 = lo[1] + (int)((t / ext[2]) % ext[1]);
        const int c0 = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        adj_grid_node(P, pm, grid_v_adj, pm_adj, node_index(c0, c1, c2, P.R), c0, c1, c2, true);
    }
}

// ---------------------------------------------------------------- P2G
// tau is the Ding state stress, or the neo-Hookean stress of F.
template <bool kLoaf = false>
__global__ void __launch_bounds__(kThreads) k_adj_p2g(AdjParams P, BkState in, const float* __restrict__ mass,
                                                   const float* __restrict__ volume, const float4* __restrict__ pm_adj,
                                                   AdjState in_adj, double* __restrict__ params_adj) {
    if constexpr (kLoaf) fix_loaf_mode(P);
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    float acc_mu = 0.f, acc_lam = 0.f;
    if (i < P.n) {
        const int64_t pitch = P.pitch;
        V3 xi = load_v3(in.x, i, pitch);
        Stencil st = make_stencil(xi, P.origin, P.dx, P.R);
        if (st.valid) {
            float m = mass[i];
            float scale = P.dt * volume[i] * 4.0f / (P.dx * P.dx);
            M3 Cm = load_m3(in.C, i, pitch);
            M3 F = load_m3(in.F, i, pitch);
            M3 tau;
            float J = det3(F);
            if (P.material == 1) {
                tau = load_m3(in.tau, i, pitch);
            } else {
                float lj = logf(J);
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float ffT = F.m[3 * r] * F.m[3 * c] + F.m[3 * r + 1] * F.m[3 * c + 1] + F.m[3 * r + 2] * F.m[3 * c + 2];
                        float id = r == c ? 1.f : 0.f;
                        tau.m[3 * r + c] = P.ding.mu * (ffT - id) + P.ding.lam * lj * id;
                    }
            }
            V3 vel = load_v3(in.v, i, pitch);
            float A[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) A[e] = m * Cm.m[e] - scale * tau.m[e];
            float vb[3] = {0.f, 0.f, 0.f}, Ab[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            float xg[3] = {0.f, 0.f, 0.f}, mb = 0.f;
            const float inv_dx = 1.f / P.dx;
#pragma unroll
            for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                    for (int oz = 0; oz < 3; ++oz) {
                        const int o[3] = {ox, oy, oz};
                        float wa[3] = {st.w[0][ox], st.w[1][oy], st.w[2][oz]};
                        float w = wa[0] * wa[1] * wa[2];
                        float d[3] = {((float)ox - st.l[0]) * P.dx, ((float)oy - st.l[1]) * P.dx, ((float)oz - st.l[2]) * P.dx};
                        float4 g = __ldg(pm_adj + node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R));
                        float pb[3] = {g.x, g.y, g.z};
                        float Ad[3];
#pragma unroll
                        for (int r = 0; r < 3; ++r) Ad[r] = A[3 * r] * d[0] + A[3 * r + 1] * d[1] + A[3 * r + 2] * d[2];
                        // node mass w m, momentum w (m v + A d)
#pragma unroll
                        for (int r = 0; r < 3; ++r) {
                            vb[r] += w * m * pb[r];
#pragma unroll
                            for (int c = 0; c < 3; ++c) Ab[3 * r + c] += w * pb[r] * d[c];
                        }
                        float sdot = g.w * m + pb[0] * (m * vel.v[0] + Ad[0]) + pb[1] * (m * vel.v[1] + Ad[1]) +
                                     pb[2] * (m * vel.v[2] + Ad[2]);
                        // node mass w m and momentum w m (v + C d): the particle-mass adjoint
                        float Cd[3];
#pragma unroll
                        for (int r = 0; r < 3; ++r) Cd[r] = Cm.m[3 * r] * d[0] + Cm.m[3 * r + 1] * d[1] + Cm.m[3 * r + 2] * d[2];
                        mb += w * (g.w + pb[0] * (vel.v[0] + Cd[0]) + pb[1] * (vel.v[1] + Cd[1]) + pb[2] * (vel.v[2] + Cd[2]));
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            float dw = qweight_grad(st.l[a], o[a]) * inv_dx;
                            float rest = 1.f;
#pragma unroll
                            for (int b2 = 0; b2 < 3; ++b2)
                                if (b2 != a) rest *= wa[b2];
                            // d = x_i - x_p: dd/dx_p = -I, so A d contributes -w A^T pb
                            float atp = A[a] * pb[0] + A[3 + a] * pb[1] + A[6 + a] * pb[2];
                            xg[a] += dw * rest * sdot - w * atp;
                        }
                    }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                in_adj.x[c * pitch + i] += xg[c];
                in_adj.v[c * pitch + i] = vb[c];
            }
            if (in_adj.mass) in_adj.mass[i] = mb;
            // A = m C - scale tau
            float Cb[9], taub[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) {
                Cb[e] = m * Ab[e];
                taub[e] = -scale * Ab[e];
            }
#pragma unroll
            for (int e = 0; e < 9; ++e) in_adj.C[e * pitch + i] = Cb[e];
            if (P.material == 1) {
#pragma unroll
                for (int e = 0; e < 9; ++e) in_adj.tau[e * pitch + i] = taub[e];
            } else {
                // tau = mu (F F^T - I) + lam log J I
                float Fb[9];
                M3 inv = inverse3(F);
                float trb = taub[0] + taub[4] + taub[8];
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float t = 0.f;
#pragma unroll
                        for (int k = 0; k < 3; ++k) t += (taub[3 * r + k] + taub[3 * k + r]) * F.m[3 * k + c];
                        Fb[3 * r + c] = P.ding.mu * t + P.ding.lam * trb * inv.m[3 * c + r];
                    }
                add_m3(in_adj.F, i, pitch, Fb);
                float lj = logf(J);
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) {
                        float ffT = F.m[3 * r] * F.m[3 * c] + F.m[3 * r + 1] * F.m[3 * c + 1] + F.m[3 * r + 2] * F.m[3 * c + 2];
                        acc_mu += taub[3 * r + c] * (ffT - (r == c ? 1.f : 0.f));
                    }
                acc_lam = trb * lj;
            }
        } else {
            if (in_adj.mass) in_adj.mass[i] = 0.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) in_adj.v[c * pitch + i] = 0.f;
#pragma unroll
            for (int e = 0; e < 9; ++e) in_adj.C[e * pitch + i] = 0.f;
            if (P.material == 1) {
#pragma unroll
                for (int e = 0; e < 9; ++e) in_adj.tau[e * pitch + i] = 0.f;
            }
        }
    }
    if (params_adj && P.material != 1) {
        block_accumulate(params_adj + 0, acc_mu);
        block_accumulate(params_adj + 1, acc_lam);
    }
}

AdjParams adj_params(const BkSubstepParams& p) {
    AdjParams a;
    a.n = p.n; a.pitch = p.pitch; a.R = p.resolution; a.bc = p.boundary_cells;
    for (int k = 0; k < 3; ++k) { a.origin[k] = p.origin[k]; a.gravity[k] = p.gravity[k]; }
    a.dx = p.spacing; a.dt = p.time_step;
    a.material = p.material;
    a.transport = p.transport;
    const BkDingParams& d = p.ding;
    a.ding.coupled_porosity = d.coupled_porosity; a.ding.temperature_enabled = d.temperature_enabled;
    a.ding.mu = d.shear_modulus; a.ding.lam = d.lame_lambda; a.ding.yield_stress = d.yield_stress;
    a.ding.initial_porosity = d.initial_porosity; a.ding.dt = d.time_step;
    for (int k = 0; k < 4; ++k) {
        a.ding.knots[k] = d.temperature_knots[k];
        a.ding.yield_factors[k] = d.yield_factors[k];
        a.ding.viscosity_factors[k] = d.viscosity_factors[k];
    }
    return a;
}

AdjState adj_state(const BkAdjointState& s) {
    AdjState a;
    a.x = s.x; a.v = s.v; a.C = s.C; a.F = s.F; a.Fe = s.Fe; a.tau = s.tau; a.porosity = s.porosity;
    a.temperature = s.temperature;
    a.mass = s.mass;
    return a;
}

}  // namespace

extern "C" {

int bk_substep_adjoint(const BkSubstepParams* params, const BkState* in, const BkConstants* constants,
                       const float* node_pm, const float* node_v, const int32_t* node_box,
                       const BkAdjointState* out_adjoint, BkAdjointState* in_adjoint, float* node_v_adjoint,
                       float* node_pm_adjoint, double* parameter_adjoint, void* stream) {
    if (!params || !in || !constants || !node_pm || !node_v || !out_adjoint || !in_adjoint || !node_v_adjoint ||
        !node_pm_adjoint)
        return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: null argument");
    const BkSubstepParams& p = *params;
    if (p.gas && !p.transport)
        return bk::fail(BK_ERR_UNSUPPORTED, "bk_substep_adjoint: gas mode runs with transport");
    if (p.transport && p.material != 1)
        return bk::fail(BK_ERR_UNSUPPORTED, "bk_substep_adjoint: with transport the adjoint needs the Ding model");
    if (p.n < 0 || p.pitch < p.n || p.resolution < 4) return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: bad sizes");
    if (p.material == 1 && (!in->Fe || !in->tau || !in->porosity || !in->gelled ||
                            !in->material_temperature || !out_adjoint->Fe || !in_adjoint->Fe ||
                            !constants->viscosity_parameter))
        return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: missing Ding arrays");
    if (!constants->mass || !constants->volume) return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: missing constants");
    if (p.n == 0) return BK_OK;
    AdjParams a = adj_params(p);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t nodes = (int64_t)p.resolution * p.resolution * p.resolution;
    if (!node_box) cudaMemsetAsync(node_v_adjoint, 0, nodes * sizeof(float4), s);
    unsigned blocks = (unsigned)((p.n + kThreads - 1) / kThreads);
    const bool loaf = adj_loaf_mode(p);
    const bool coupled = p.material == 1 && p.ding.coupled_porosity;
    auto* g2p_return = coupled ? (loaf ? k_adj_g2p_return<true, true> : k_adj_g2p_return<true>)
                               : (loaf ? k_adj_g2p_return<false, true> : k_adj_g2p_return<false>);
    g2p_return<<<blocks, kThreads, 0, s>>>(a, *in, reinterpret_cast<const float4*>(node_v),
                                           constants->viscosity_parameter, adj_state(*out_adjoint),
                                           adj_state(*in_adjoint), parameter_adjoint);
    if (int rc = bk::check_launch("bk_substep_adjoint/g2p_return")) return rc;
    (loaf ? k_adj_g2p_scatter<true> : k_adj_g2p_scatter<false>)<<<blocks, kThreads, 0, s>>>(
        a, *in, reinterpret_cast<const float4*>(node_v), adj_state(*out_adjoint), adj_state(*in_adjoint),
        reinterpret_cast<float4*>(node_v_adjoint));
    if (int rc = bk::check_launch("bk_substep_adjoint/g2p_scatter")) return rc;
    if (node_box) {
        int device = 0, sms = 148;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        k_adj_grid_box<<<(unsigned)sms * 4, 256, 0, s>>>(a, node_box, reinterpret_cast<const float4*>(node_pm),
                                                          reinterpret_cast<float4*>(node_v_adjoint),
                                                          reinterpret_cast<float4*>(node_pm_adjoint));
    } else {
        k_adj_grid<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(a, reinterpret_cast<const float4*>(node_pm),
                                                                  reinterpret_cast<float4*>(node_v_adjoint),
                                                                  reinterpret_cast<float4*>(node_pm_adjoint), nodes);
    }
    if (int rc = bk::check_launch("bk_substep_adjoint/grid")) return rc;
    (loaf ? k_adj_p2g<true> : k_adj_p2g<false>)<<<blocks, kThreads, 0, s>>>(a, *in, constants->mass, constants->volume,
                                          reinterpret_cast<const float4*>(node_pm_adjoint), adj_state(*in_adjoint),
                                          parameter_adjoint);
    return bk::check_launch("bk_substep_adjoint/p2g");
}

}  // extern "C"
