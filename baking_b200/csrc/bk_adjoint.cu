// Hand-written adjoint of the mechanics substep (P2G -> grid update -> G2P -> return map).
//
// Reverse order of one substep t -> t+1, given the adjoint of state t+1 and the forward grid of step
// t (node mass, momentum and velocity, recomputed by the caller from the checkpointed state t):
//
//   adj_g2p_return   per particle: recompute G2P and the return map, then pull the adjoints of
//                    x', v', C', F', Fe', tau', porosity' back to x, F, Fe, porosity, temperature and
//                    the material parameters; scatter the grid-velocity adjoint.
//   adj_grid         per node: velocity adjoint -> momentum and mass adjoints (walls clamp to zero).
//   adj_p2g          per particle: gather the momentum/mass adjoints -> v, C, tau (and, for the
//                    neo-Hookean model, F and mu, lambda) and the weight-gradient terms of x.
//
// The return map's backward uses the derivative of isotropic matrix functions: with trial
// A = U diag(s) V^T, Fe' = U diag(g(s)) V^T and tau' = U diag(h(s)) U^T, the off-diagonal terms
// in the rotated frame use divided differences of g and h. For this model they have closed
// forms (g_j - g_i and h_j - h_i depend on log(s_j / s_i) alone), evaluated with expm1/log1p so
// they stay finite as two singular values coincide. The diagonal and parameter derivatives come
// from forward-mode duals through the principal-space chain, including the implicit overstress
// solve (derivatives as in the reference's SolveOverstressGradient, ding.py:90-100).
// Differentiable parameters: shear modulus, Lame lambda, the viscosity parameter and the
// per-particle temperature (through the yield and viscosity factor tables). The gelation latch and
// the wall and stencil switches are discrete; like the reference, no gradient flows through them.
#include <climits>
#include <cstdio>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"
#include "bk_dual.cuh"

using namespace bk;

namespace {

constexpr int kThreads = 128;

struct AdjParams {
    int64_t n, pitch;
    int R, bc;
    float origin[3], dx, dt, gravity[3];
    int material;  // 0 neo-Hookean, 1 Ding
    DingParamsDev ding;
};

// Adjoint of a particle state: same planes as BkState.
struct AdjState {
    float *x, *v, *C, *F, *Fe, *tau, *porosity, *temperature;
};

// Directional-derivative slots of the principal-space duals.
enum { kS0 = 0, kS1, kS2, kMu, kLam, kTy, kEta, kA, kDirs };
using D8 = Dual<kDirs>;

struct Principal {
    float g[3], h[3];          // Fe' = U diag(g) V^T, tau' = U diag(h) U^T
    float dg[3][kDirs], dh[3][kDirs];
    float r, df;               // overstress root and deviatoric factor d
    float iso;                 // common isochoric factor applied to g (1 when a != 0)
};

// sigma -> (g, h) of the Ding return map (ding.py:103-131) with derivatives.
__device__ Principal principal(const float* s, float mu, float lam, float ty, float eta, float a, float dt) {
    D8 S[3] = {D8::seed(s[0], kS0), D8::seed(s[1], kS1), D8::seed(s[2], kS2)};
    D8 Mu = D8::seed(mu, kMu), Lam = D8::seed(lam, kLam), Ty = D8::seed(ty, kTy), Eta = D8::seed(eta, kEta);
    D8 Aa = D8::seed(a, kA);
    D8 eps[3] = {dlog(S[0]), dlog(S[1]), dlog(S[2])};
    D8 tr = eps[0] + eps[1] + eps[2];
    D8 two_mu = scale(Mu, 2.f);
    D8 ts[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ts[k] = two_mu * eps[k] + Lam * tr;
    D8 mean = scale(ts[0] + ts[1] + ts[2], 1.f / 3.f);
    D8 dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
    D8 ty2 = Ty * Ty;
    D8 q2 = scale(dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2], 1.5f) / ty2;
    D8 p2 = Aa * mean * mean / ty2;
    D8 bulk = two_mu + scale(Lam, 3.f);
    D8 d = scale(Mu, 6.f * dt) * ty2 / Eta;
    D8 h = scale(Aa, 2.f / 3.f * dt) * bulk * ty2 / Eta;
    float r = solve_overstress(q2.v, p2.v, d.v, h.v);
    D8 R(r);
    if (q2.v + p2.v > 1.0f) {
        // R(r) = r + 1 - q2/(1+dr)^2 - p2/(1+hr)^2 = 0: dr = -(R_q2 dq2 + R_p2 dp2 + R_d dd + R_h dh) / R_r.
        float u = 1.f + d.v * r, w = 1.f + h.v * r;
        float Rr = 1.f + 2.f * d.v * q2.v / (u * u * u) + 2.f * h.v * p2.v / (w * w * w);
        float Rq = -1.f / (u * u), Rp = -1.f / (w * w);
        float Rd = 2.f * q2.v * r / (u * u * u), Rh = 2.f * p2.v * r / (w * w * w);
#pragma unroll
        for (int k = 0; k < kDirs; ++k) R.d[k] = -(Rq * q2.d[k] + Rp * p2.d[k] + Rd * d.d[k] + Rh * h.d[k]) / Rr;
    }
    D8 one(1.f);
    D8 cs[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) cs[k] = dev[k] / (one + d * R) + mean / (one + h * R);
    D8 cm = scale(cs[0] + cs[1] + cs[2], 1.f / 3.f);
    D8 g[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) g[k] = dexp((cs[k] - cm) / two_mu + cm / bulk);
    Principal out;
    out.iso = 1.f;
    if (a == 0.0f) {
        // Isochoric correction (ding.py:129-131): Fe' *= cbrt(det trial / det Fe'), a common factor.
        D8 c = dcbrt((S[0] * S[1] * S[2]) / (g[0] * g[1] * g[2]));
        out.iso = c.v;
#pragma unroll
        for (int k = 0; k < 3; ++k) g[k] = g[k] * c;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        out.g[k] = g[k].v;
        out.h[k] = cs[k].v;
#pragma unroll
        for (int j = 0; j < kDirs; ++j) {
            out.dg[k][j] = g[k].d[j];
            out.dh[k][j] = cs[k].d[j];
        }
    }
    out.r = r;
    out.df = d.v;
    return out;
}

// expm1(x / c) / expm1(x), finite at x = 0.
__device__ __forceinline__ float ratio_expm1(float x, float c) {
    if (fabsf(x) < 1e-12f) return 1.f / c;
    return expm1f(x / c) / expm1f(x);
}

// x / expm1(x), finite at x = 0.
__device__ __forceinline__ float x_over_expm1(float x) {
    if (fabsf(x) < 1e-12f) return 1.f;
    return x / expm1f(x);
}

__device__ __forceinline__ void add_m3(float* __restrict__ p, int64_t i, int64_t pitch, const float* a) {
#pragma unroll
    for (int c = 0; c < 9; ++c) p[c * pitch + i] += a[c];
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
__global__ void __launch_bounds__(kThreads) k_adj_g2p_return(AdjParams P, BkState in, const float4* __restrict__ grid_v,
                                                          const float* __restrict__ eta_param, AdjState out_adj,
                                                          AdjState in_adj, float4* __restrict__ grid_v_adj,
                                                          double* __restrict__ params_adj) {
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    float acc_mu = 0.f, acc_lam = 0.f, acc_eta = 0.f;
    if (i < P.n) {
        const int64_t pitch = P.pitch;
        V3 xi = load_v3(in.x, i, pitch);
        Stencil st = make_stencil(xi, P.origin, P.dx, P.R);
        if (st.valid) {
            // ---- forward recompute: G2P
            float nv[3] = {0.f, 0.f, 0.f}, nc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
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
                        for (int r = 0; r < 3; ++r) {
                            nv[r] += w * uu[r];
#pragma unroll
                            for (int c = 0; c < 3; ++c) nc[3 * r + c] += k4 * w * (uu[r] * d[c]);
                        }
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
                Tb = out_adj.temperature[i];
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
                float s[3];
                svd3f(trial, U, s, V);
                float a = porosity_coefficient(por);
                Principal pr = principal(s, D.mu, D.lam, ty, eta, a, D.dt);
                // porosity' = det(F') / prod(g) - 1 + n0 (uncoupled; zero when n0 = n = 0)
                float prod_g = pr.g[0] * pr.g[1] * pr.g[2];
                bool porosity_free = !(D.initial_porosity == 0.0f && por == 0.0f);
                float detFn = det3(Fn);
                float gb_por[3] = {0.f, 0.f, 0.f};
                if (porosity_free && por_b != 0.f) {
                    float npor = detFn / prod_g;
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
                // rotated adjoints
                float Gh[9], Th[9];
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        float gs = 0.f, tsum = 0.f;
#pragma unroll
                        for (int r = 0; r < 3; ++r)
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                gs += U.m[3 * r + p] * Fe_b[3 * r + c] * V.m[3 * c + q];
                                tsum += U.m[3 * r + p] * tau_b[3 * r + c] * U.m[3 * c + q];
                            }
                        Gh[3 * p + q] = gs;
                        Th[3 * p + q] = tsum;
                    }
                // diagonal: sbar_j = sum_i (Gh_ii + gb_por_i) dg_i/ds_j + Th_ii dh_i/ds_j; parameters likewise
                float Ab[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
                float dpar[kDirs];
#pragma unroll
                for (int j = 0; j < kDirs; ++j) {
                    float t = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k) t += (Gh[4 * k] + gb_por[k]) * pr.dg[k][j] + Th[4 * k] * pr.dh[k][j];
                    dpar[j] = t;
                }
                Ab[0] = dpar[kS0];
                Ab[4] = dpar[kS1];
                Ab[8] = dpar[kS2];
                // off-diagonal: divided differences in closed form
                const float one_dr = 1.f + pr.df * pr.r;
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        if (p == q) continue;
                        // pair (i=p, j=q): L = log(s_q / s_p)
                        float L = log1pf((s[q] - s[p]) / s[p]);
                        // dFe^_pq = P_pq M_pq + Q_pq M_qp with M = U^T dA V,
                        //   P_pq = (g_q s_q - g_p s_p) / (s_q^2 - s_p^2), Q_pq = (g_q s_p - g_p s_q) / (s_q^2 - s_p^2);
                        // dtau^_pq = D_pq (s_q M_pq + s_p M_qp), D_pq = (h_q - h_p) / (s_q^2 - s_p^2).
                        // g_q / g_p = exp(L / (1 + d r)) and h_q - h_p = 2 mu L / (1 + d r).
                        float ddg = (pr.g[p] / s[p]) * ratio_expm1(L, one_dr);  // (g_q - g_p) / (s_q - s_p)
                        float P_pq = (ddg * s[q] + pr.g[p]) / (s[q] + s[p]);
                        float ddg_r = (pr.g[q] / s[q]) * ratio_expm1(-L, one_dr);  // (g_p - g_q) / (s_p - s_q)
                        float Q_qp = (ddg_r * s[q] - pr.g[q]) / (s[p] + s[q]);
                        float D_pq = 2.f * D.mu / (one_dr * (s[q] + s[p]) * s[p]) * x_over_expm1(L);
                        Ab[3 * p + q] = Gh[3 * p + q] * P_pq + Gh[3 * q + p] * Q_qp +
                                        (Th[3 * p + q] + Th[3 * q + p]) * D_pq * s[q];
                    }
                // trial adjoint A_bar = U Ab V^T
                float Tb_m[9];
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float t = 0.f;
#pragma unroll
                        for (int p = 0; p < 3; ++p)
#pragma unroll
                            for (int q = 0; q < 3; ++q) t += U.m[3 * r + p] * Ab[3 * p + q] * V.m[3 * c + q];
                        Tb_m[3 * r + c] = t;
                    }
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
                // porosity -> a(n) (zero at n = 0)
                if (por > 0.0f) {
                    float lg = logf(1.0f / por);
                    float da = a * (2.0f / (por * lg) - 3.5f / (3.5f * por + 1.0f));
                    porb_in = dpar[kA] * da;
                }
            }
            // ---- G2P backward
            // x' = x + dt v'; F' = (I + dt C') F
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
            // v' = sum w v_i; C' = k sum w v_i d^T with d = x_i - x_p
            float xg[3] = {xb[0], xb[1], xb[2]};
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
                        int64_t node = node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R);
                        float4 u = __ldg(grid_v + node);
                        float uu[3] = {u.x, u.y, u.z};
                        // node velocity adjoint: w (vb + k Cb d)
                        float nb[3];
#pragma unroll
                        for (int r = 0; r < 3; ++r)
                            nb[r] = w * (vb[r] + k4 * (Cb[3 * r] * d[0] + Cb[3 * r + 1] * d[1] + Cb[3 * r + 2] * d[2]));
                        atomicAdd(grid_v_adj + node, make_float4(nb[0], nb[1], nb[2], 0.f));
                        // scalar s = vb . u + k u^T Cb d  (the weight's cofactor)
                        float sdot = vb[0] * uu[0] + vb[1] * uu[1] + vb[2] * uu[2];
                        float cu[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) cu[c] = Cb[c] * uu[0] + Cb[3 + c] * uu[1] + Cb[6 + c] * uu[2];
                        sdot += k4 * (cu[0] * d[0] + cu[1] * d[1] + cu[2] * d[2]);
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            float dw = qweight_grad(st.l[a], o[a]) * inv_dx;
                            float rest = 1.f;
#pragma unroll
                            for (int b2 = 0; b2 < 3; ++b2)
                                if (b2 != a) rest *= wa[b2];
                            xg[a] += dw * rest * sdot - k4 * w * cu[a];  // d = x_i - x_p: dd/dx_p = -I
                        }
                    }
            store_v3(in_adj.x, i, pitch, V3{{xg[0], xg[1], xg[2]}});
            // F, C (of state t) adjoints: F from G2P; C gets no direct dependence from G2P (C' does)
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
            // The forward raised the stencil flag for this particle; its adjoint is zero.
#pragma unroll
            for (int c = 0; c < 3; ++c) in_adj.x[c * pitch + i] = 0.f;
#pragma unroll
            for (int c = 0; c < 9; ++c) in_adj.F[c * pitch + i] = 0.f;
            if (P.material == 1) {
#pragma unroll
                for (int c = 0; c < 9; ++c) in_adj.Fe[c * pitch + i] = 0.f;
                in_adj.porosity[i] = 0.f;
                in_adj.temperature[i] = out_adj.temperature[i];
            }
        }
    }
    if (params_adj) {
        block_accumulate(params_adj + 0, acc_mu);
        block_accumulate(params_adj + 1, acc_lam);
        block_accumulate(params_adj + 2, acc_eta);
    }
}

// ------------------------------------------------------------- grid update
__global__ void k_adj_grid(AdjParams P, const float4* __restrict__ pm, const float4* __restrict__ grid_v_adj,
                           float4* __restrict__ pm_adj, int64_t nodes) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    float4 a = grid_v_adj[i];
    float4 q = pm[i];
    float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
    if (q.w > 0.0f && (a.x != 0.f || a.y != 0.f || a.z != 0.f)) {
        const int R = P.R, bc = P.bc;
        int c[3] = {(int)(i / ((int64_t)R * R)), (int)((i / R) % R), (int)(i % R)};
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
}

// ---------------------------------------------------------------- P2G
// tau is the Ding state stress, or the neo-Hookean stress of F.
__global__ void __launch_bounds__(kThreads) k_adj_p2g(AdjParams P, BkState in, const float* __restrict__ mass,
                                                   const float* __restrict__ volume, const float4* __restrict__ pm_adj,
                                                   AdjState in_adj, double* __restrict__ params_adj) {
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
            float xg[3] = {0.f, 0.f, 0.f};
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
    return a;
}

}  // namespace

extern "C" {

int bk_substep_adjoint(const BkSubstepParams* params, const BkState* in, const BkConstants* constants,
                       const float* node_pm, const float* node_v, const BkAdjointState* out_adjoint,
                       BkAdjointState* in_adjoint, float* node_v_adjoint, float* node_pm_adjoint,
                       double* parameter_adjoint, void* stream) {
    if (!params || !in || !constants || !node_pm || !node_v || !out_adjoint || !in_adjoint || !node_v_adjoint ||
        !node_pm_adjoint)
        return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: null argument");
    const BkSubstepParams& p = *params;
    if (p.transport || p.gas)
        return bk::fail(BK_ERR_UNSUPPORTED, "bk_substep_adjoint: the adjoint covers the mechanics substep (no transport/gas)");
    if (p.n < 0 || p.pitch < p.n || p.resolution < 4) return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: bad sizes");
    if (p.material == 1 && (p.ding.coupled_porosity || !in->Fe || !in->tau || !in->porosity || !in->gelled ||
                            !in->material_temperature || !out_adjoint->Fe || !in_adjoint->Fe ||
                            !constants->viscosity_parameter))
        return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: missing Ding arrays");
    if (!constants->mass || !constants->volume) return bk::fail(BK_ERR_ARGUMENT, "bk_substep_adjoint: missing constants");
    if (p.n == 0) return BK_OK;
    AdjParams a = adj_params(p);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int64_t nodes = (int64_t)p.resolution * p.resolution * p.resolution;
    cudaMemsetAsync(node_v_adjoint, 0, nodes * sizeof(float4), s);
    unsigned blocks = (unsigned)((p.n + kThreads - 1) / kThreads);
    k_adj_g2p_return<<<blocks, kThreads, 0, s>>>(a, *in, reinterpret_cast<const float4*>(node_v),
                                                 constants->viscosity_parameter, adj_state(*out_adjoint),
                                                 adj_state(*in_adjoint), reinterpret_cast<float4*>(node_v_adjoint),
                                                 parameter_adjoint);
    if (int rc = bk::check_launch("bk_substep_adjoint/g2p_return")) return rc;
    k_adj_grid<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(a, reinterpret_cast<const float4*>(node_pm),
                                                              reinterpret_cast<const float4*>(node_v_adjoint),
                                                              reinterpret_cast<float4*>(node_pm_adjoint), nodes);
    if (int rc = bk::check_launch("bk_substep_adjoint/grid")) return rc;
    k_adj_p2g<<<blocks, kThreads, 0, s>>>(a, *in, constants->mass, constants->volume,
                                          reinterpret_cast<const float4*>(node_pm_adjoint), adj_state(*in_adjoint),
                                          parameter_adjoint);
    return bk::check_launch("bk_substep_adjoint/p2g");
}

}  // extern "C"
