// One sm_100a kernel per reference Warp kernel, behind the C ABI of include/baking_b200.h.
//
// These are the kernel-level entry points (the reference's `wp.launch(Kernel, ...)`
// calls); the simulator's substep uses the fused kernels of bk_substep.cu, which call
// the same device functions. Layout: structure-of-arrays planes (see the header).
#include <cstdio>
#include <cstring>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"

using namespace bk;

namespace {
thread_local char g_error[512] = "";
}

int bk::fail(int code, const char* msg) {
    snprintf(g_error, sizeof g_error, "%s", msg);
    return code;
}

int bk::check_launch(const char* name) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_error, sizeof g_error, "%s: %s", name, cudaGetErrorString(e));
        return BK_ERR_LAUNCH;
    }
    return BK_OK;
}

namespace {

constexpr int kBlock = 256;

inline unsigned blocks_for(int64_t n, int block = kBlock) { return (unsigned)((n + block - 1) / block); }

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

struct Origin { float o[3]; };

inline Origin origin_of(const float* o) { Origin r{}; if (o) { r.o[0] = o[0]; r.o[1] = o[1]; r.o[2] = o[2]; } return r; }

// ------------------------------------------------------- transfer.py:36-70
__global__ void k_particle_to_grid(int64_t n, int64_t pitch, const float* __restrict__ x, const float* __restrict__ v,
                                   const float* __restrict__ C, const float* __restrict__ tau,
                                   const float* __restrict__ mass, const float* __restrict__ V0,
                                   float4* __restrict__ node_pm, Origin origin, float dx, int R, float dt,
                                   int32_t* flags) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stencil st = make_stencil(load_v3(x, i, pitch), origin.o, dx, R);
    if (!st.valid) { set_flag(flags, 1); return; }
    float m = mass[i];
    float scale = dt * V0[i] * 4.0f / (dx * dx);
    M3 Cm = load_m3(C, i, pitch), T = load_m3(tau, i, pitch);
    float A[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) A[e] = m * Cm.m[e] - scale * T.m[e];
    V3 vel = load_v3(v, i, pitch);
    float mv[3] = {m * vel.v[0], m * vel.v[1], m * vel.v[2]};
#pragma unroll
    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                float w = st.w[0][ox] * st.w[1][oy] * st.w[2][oz];
                float d[3] = {((float)ox - st.l[0]) * dx, ((float)oy - st.l[1]) * dx, ((float)oz - st.l[2]) * dx};
                float4 add;
                add.x = w * (mv[0] + (A[0] * d[0] + A[1] * d[1] + A[2] * d[2]));
                add.y = w * (mv[1] + (A[3] * d[0] + A[4] * d[1] + A[5] * d[2]));
                add.z = w * (mv[2] + (A[6] * d[0] + A[7] * d[1] + A[8] * d[2]));
                add.w = w * m;
                atomicAdd(node_pm + node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, R), add);
            }
}

// --------------------------------------------------------- grid.py:20-38
__global__ void k_update_grid(int R, const float4* __restrict__ node_pm, float4* __restrict__ node_v, int bc,
                              float gx, float gy, float gz, float dt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t nn = (int64_t)R * R * R;
    if (i >= nn) return;
    float4 pm = node_pm[i];
    if (!(pm.w > 0.0f)) return;
    float vel[3] = {pm.x / pm.w + dt * gx, pm.y / pm.w + dt * gy, pm.z / pm.w + dt * gz};
    int c[3] = {(int)(i / ((int64_t)R * R)), (int)((i / R) % R), (int)(i % R)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (c[a] < bc && vel[a] < 0.0f) vel[a] = 0.0f;
        if (c[a] >= R - bc && vel[a] > 0.0f) vel[a] = 0.0f;
    }
    node_v[i] = make_float4(vel[0], vel[1], vel[2], 0.0f);
}

// ------------------------------------------------------ transfer.py:73-109
__global__ void k_grid_to_particle(int64_t n, int64_t pitch, const float* __restrict__ x_in,
                                   const float* __restrict__ F_in, const float4* __restrict__ node_v,
                                   float* __restrict__ x_out, float* __restrict__ v_out, float* __restrict__ C_out,
                                   float* __restrict__ F_out, Origin origin, float dx, int R, float dt,
                                   int32_t* flags) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    V3 xi = load_v3(x_in, i, pitch);
    Stencil st = make_stencil(xi, origin.o, dx, R);
    if (!st.valid) { set_flag(flags, 1); return; }
    float nv[3] = {0, 0, 0}, nc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const float k = 4.0f / (dx * dx);
#pragma unroll
    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                float w = st.w[0][ox] * st.w[1][oy] * st.w[2][oz];
                float d[3] = {((float)ox - st.l[0]) * dx, ((float)oy - st.l[1]) * dx, ((float)oz - st.l[2]) * dx};
                float4 u = __ldg(node_v + node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, R));
                float uu[3] = {u.x, u.y, u.z};
                float kw = k * w;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    nv[r] += w * uu[r];
#pragma unroll
                    for (int c = 0; c < 3; ++c) nc[3 * r + c] += kw * (uu[r] * d[c]);
                }
            }
    M3 F = load_m3(F_in, i, pitch);
    M3 G;
#pragma unroll
    for (int e = 0; e < 9; ++e) G.m[e] = dt * nc[e] + ((e % 4) == 0 ? 1.0f : 0.0f);
    M3 Fn = matmul(G, F);
    V3 vo{{nv[0], nv[1], nv[2]}}, xo{{xi.v[0] + dt * nv[0], xi.v[1] + dt * nv[1], xi.v[2] + dt * nv[2]}};
    store_v3(v_out, i, pitch, vo);
    M3 Co;
#pragma unroll
    for (int e = 0; e < 9; ++e) Co.m[e] = nc[e];
    store_m3(C_out, i, pitch, Co);
    store_v3(x_out, i, pitch, xo);
    store_m3(F_out, i, pitch, Fn);
}

// ---------------------------------------------------- elastic.py:4-26
__global__ void k_elastic_stress(int64_t n, int64_t pitch, const float* __restrict__ Fp, float* __restrict__ tau,
                                 float mu, float lam, int32_t* flags) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    M3 F = load_m3(Fp, i, pitch);
    float J = det3(F);
    M3 t;
    if (!isfinite(J) || J <= 0.0f) {
        set_flag(flags, 0);
#pragma unroll
        for (int e = 0; e < 9; ++e) t.m[e] = 0.0f;
    } else {
        float lj = logf(J);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float ffT = F.m[3 * r] * F.m[3 * c] + F.m[3 * r + 1] * F.m[3 * c + 1] + F.m[3 * r + 2] * F.m[3 * c + 2];
                float id = r == c ? 1.0f : 0.0f;
                t.m[3 * r + c] = mu * (ffT - id) + lam * lj * id;
            }
    }
    store_m3(tau, i, pitch, t);
}

// ---------------------------------------------------- ding.py:140-221
__global__ void k_update_ding(int64_t n, int64_t pitch, const float* __restrict__ Fe_old,
                              const float* __restrict__ por_old, const int32_t* __restrict__ gel_old,
                              const float* __restrict__ F_tot, const float* __restrict__ C_new,
                              float* __restrict__ Fe_new, float* __restrict__ Fp_new, float* __restrict__ tau_new,
                              float* __restrict__ residuals, float* __restrict__ por_new, float* __restrict__ T_out,
                              int32_t* __restrict__ gel_new, float* __restrict__ yield_out,
                              float* __restrict__ visc_out, const float* __restrict__ eta_param, int32_t* flags,
                              float* __restrict__ por_res, DingParamsDev P, const float* __restrict__ T_local) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    DingParticleOut o;
    float T = T_local[i];
    if (!update_ding_particle(P, load_m3(Fe_old, i, pitch), por_old[i], gel_old[i], load_m3(F_tot, i, pitch),
                              load_m3(C_new, i, pitch), T, __ldg(eta_param), flags, o))
        return;
    store_m3(Fe_new, i, pitch, o.Fe);
    store_m3(Fp_new, i, pitch, o.Fp);
    store_m3(tau_new, i, pitch, o.tau);
    residuals[i] = o.residual;
    por_res[i] = o.porosity_residual;
    por_new[i] = o.porosity;
    T_out[i] = T;
    gel_new[i] = o.gelled;
    yield_out[i] = o.yield_stress;
    visc_out[i] = o.viscosity;
}

// -------------------------------------------------------- gas.py:16-45
__global__ void k_combine_gas_stress(int64_t n, int64_t pitch, const float* __restrict__ tau_s,
                                     const float* __restrict__ Fp, const float* __restrict__ por,
                                     const double* __restrict__ moles, const float* __restrict__ T,
                                     float* __restrict__ tau_t, int32_t* flags, float ambient, float n0,
                                     const float* __restrict__ density, float K, float dt, float dx, float cfl) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float J = det3(load_m3(Fp, i, pitch));
    float ni = por[i];
    if (ni <= 0.0f || ni >= 1.0f || !isfinite(ni) || J <= 0.0f) { set_flag(flags, 0); return; }
    float p = (float)gas_pressure(moles[i], T[i], J, ni);
    float iso = J * (ambient - p);
    M3 t = load_m3(tau_s, i, pitch);
#pragma unroll
    for (int e = 0; e < 9; ++e) t.m[e] += (e % 4) == 0 ? iso : iso * 0.0f;
    store_m3(tau_t, i, pitch, t);
    float bulk = p * (1.0f + (1.0f - n0 + ni) / ni);
    float wave = sqrtf((K + bulk) * J / density[i]);
    if (!isfinite(p) || wave * dt / dx > cfl) set_flag(flags, 2);
}

__global__ void k_refresh_gas(int64_t n, int64_t pitch, const double* __restrict__ old_moles,
                              double* __restrict__ new_moles, const float* __restrict__ Fp,
                              const float* __restrict__ por, double* __restrict__ pressures,
                              const float* __restrict__ T) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = old_moles[i];
    new_moles[i] = m;
    float ni = por[i];
    if (ni > 0.0f && ni < 1.0f) pressures[i] = gas_pressure(m, T[i], det3(load_m3(Fp, i, pitch)), ni);
}

// ----------------------------------------------- mesh_tracking.py:13-38
// One block per vertex (a vertex of a finely sampled mesh binds hundreds to thousands of particles:
// a block keeps enough of their gathers in flight and reduces the weighted sum), the block size
// chosen from the mean bindings per vertex.
template <int kVB>
__global__ void __launch_bounds__(kVB) k_reconstruct_vertices(int64_t pitch, const float* __restrict__ x,
                                                            const float* __restrict__ F, int64_t vpitch,
                                                            const float* __restrict__ ref_vertices,
                                                            const int32_t* __restrict__ offsets,
                                                            const int32_t* __restrict__ particles,
                                                            const float* __restrict__ weights, int64_t bpitch,
                                                            const float* __restrict__ ref_offsets,
                                                            float* __restrict__ out) {
    const int vtx = blockIdx.x;
    const float v = vertex_block<kVB>(offsets, particles, weights, ref_offsets, bpitch, ref_vertices, vpitch, x, F,
                                      pitch, vtx);
    if (threadIdx.x < 3) out[threadIdx.x * vpitch + vtx] = v;
}

// --------------------------------------------- thermal_water.py:77-92
__global__ void k_surface_areas(int64_t nf, int64_t vpitch, const float* __restrict__ vertices,
                                const int32_t* __restrict__ faces, const int32_t* __restrict__ owners,
                                double* exposed, double* contact, float floor_height, float contact_distance) {
    int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (f >= nf) return;
    double p[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int vtx = faces[3 * f + k];
#pragma unroll
        for (int a = 0; a < 3; ++a) p[k][a] = (double)vertices[a * vpitch + vtx];
    }
    double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    double nr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double len = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
    double area = 0.5 * len;
    double cy = (p[0][1] + p[1][1] + p[2][1]) / 3.0;
    if (cy <= (double)(floor_height + contact_distance) && nr[1] < -0.2 * len) atomicAdd(contact + owners[f], area);
    else atomicAdd(exposed + owners[f], area);
}

// --------------------------------------------- thermal_water.py:95-137
struct ScalarParamsDev {
    float oven, tray, tray_transfer, surface_loss, water_density, latent;
    int water_enabled;
    float origin[3];
    float dx;
    int R;
};

struct NodeFields { double* f[7]; };

__global__ void k_scalar_to_grid(int64_t n, int64_t pitch, const float* __restrict__ x, const float* __restrict__ Fp,
                                 const float* __restrict__ V0, const double* __restrict__ cap,
                                 const double* __restrict__ T, const double* __restrict__ W,
                                 const double* __restrict__ exposed, const double* __restrict__ contact,
                                 const float* __restrict__ heat_parameter, ScalarParamsDev P, NodeFields nf,
                                 double* __restrict__ p_heat, double* __restrict__ p_loss, int32_t* flags) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double vol = (double)V0[i] * (double)det3(load_m3(Fp, i, pitch));
    double Ti = T[i], Wi = W[i], ci = cap[i], ex = exposed[i], co = contact[i];
    double sat = Wi / ((double)P.water_density * vol);
    double loss = 0.0;
    if (P.water_enabled) loss = (double)P.surface_loss * Ti * sat * ex;
    double h = (double)__ldg(heat_parameter);
    double heat = h * ex * ((double)P.oven - Ti) + (double)P.tray_transfer * co * ((double)P.tray - Ti)
                - (double)P.latent * loss;
    double exch = h * ex + (double)P.tray_transfer * co;
    if (P.water_enabled) exch += (double)(P.latent * P.surface_loss) * sat * ex;
    p_heat[i] = heat;
    p_loss[i] = loss;
    Stencil st = make_stencil(load_v3(x, i, pitch), P.origin, P.dx, P.R);
    if (!st.valid) { set_flag(flags, 1); return; }
    double vals[7] = {vol, ci, ci * Ti, Wi, heat, loss, exch};
#pragma unroll
    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                double w = (double)(st.w[0][ox] * st.w[1][oy] * st.w[2][oz]);
                int64_t node = node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R);
                atomicAdd(nf.f[0] + node, w * vals[0]);
                atomicAdd(nf.f[1] + node, w * vals[1]);
                atomicAdd(nf.f[2] + node, w * ci * Ti);
                atomicAdd(nf.f[3] + node, w * vals[3]);
                if (ex != 0.0 || co != 0.0) {
                    atomicAdd(nf.f[4] + node, w * vals[4]);
                    atomicAdd(nf.f[5] + node, w * vals[5]);
                    atomicAdd(nf.f[6] + node, w * vals[6]);
                }
            }
}

// --------------------------------------------- thermal_water.py:140-147
__global__ void k_grid_fields(int64_t nn, const double* __restrict__ vol, const double* __restrict__ cap,
                              const double* __restrict__ energy, const double* __restrict__ water,
                              double* __restrict__ T, double* __restrict__ s, float water_density) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    double c = cap[i];
    if (c > 0.0) {
        T[i] = energy[i] / c;
        s[i] = water[i] / ((double)water_density * vol[i]);
    }
}

// --------------------------------------------- thermal_water.py:150-190
__global__ void k_diffuse_grid(int64_t nn, const double* __restrict__ vol, const double* __restrict__ cap,
                               const double* __restrict__ T, const double* __restrict__ s,
                               const double* __restrict__ water, const double* __restrict__ b_heat,
                               const double* __restrict__ b_loss, const double* __restrict__ b_exch,
                               double* __restrict__ dT, double* __restrict__ dW, int32_t* errors, float conductivity,
                               float diffusivity, float water_density, int water_enabled, float dx, int R, float dt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nn) return;
    double ci = cap[i];
    if (ci <= 0.0) return;
    int c[3] = {(int)(i / ((int64_t)R * R)), (int)((i / R) % R), (int)(i % R)};
    double heat_rate = b_heat[i], water_rate = -b_loss[i], heat_diag = b_exch[i], water_diag = 0.0;
    double vi = vol[i], Ti = T[i], si = s[i];
    const double inv_cell = (double)(dx * dx * dx);
    const double kc = (double)(conductivity * dx);
    const double kw = (double)(diffusivity * water_density * dx);
#pragma unroll
    for (int axis = 0; axis < 3; ++axis)
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            int o[3] = {c[0], c[1], c[2]};
            o[axis] += 2 * side - 1;
            if (o[axis] < 0 || o[axis] >= R) continue;
            int64_t j = node_index(o[0], o[1], o[2], R);
            if (!(cap[j] > 0.0)) continue;
            double vj = vol[j];
            double fill = 2.0 * vi * vj / (vi + vj) / inv_cell;
            double hc = kc * fill;
            double Tj = T[j];
            heat_rate += hc * (Tj - Ti);
            heat_diag += hc;
            if (water_enabled) {
                double sj = s[j];
                double mob = kw * fill * 0.5 * (Ti + Tj) * 0.5 * (si + sj);
                water_rate += mob * (sj - si);
                water_diag += mob / ((double)water_density * vi);
            }
        }
    if ((double)dt * heat_diag > ci) set_flag(errors, 0);
    double change = (double)dt * water_rate;
    if (water[i] + change < 0.0 || (double)dt * water_diag > 1.0) set_flag(errors, 1);
    dT[i] = (double)dt * heat_rate / ci;
    dW[i] = change;
}

// --------------------------------------------- thermal_water.py:193-229
__global__ void k_scalar_to_particles(int64_t n, int64_t pitch, const float* __restrict__ x,
                                      const double* __restrict__ T_old, const double* __restrict__ W_old,
                                      const double* __restrict__ loss_old, const double* __restrict__ exch_old,
                                      const double* __restrict__ dry, const float* __restrict__ V0,
                                      const float* __restrict__ Fp, const double* __restrict__ n_water,
                                      const double* __restrict__ n_dT, const double* __restrict__ n_dW,
                                      const double* __restrict__ p_heat, const double* __restrict__ p_loss,
                                      double* __restrict__ T_new, float* __restrict__ T_mat,
                                      double* __restrict__ W_new, double* __restrict__ loss_new,
                                      double* __restrict__ exch_new, float* __restrict__ mass_new,
                                      float* __restrict__ dens_new, double* __restrict__ sat_new, float rho_w,
                                      Origin origin, float dx, int R, float dt, int32_t* flags) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Stencil st = make_stencil(load_v3(x, i, pitch), origin.o, dx, R);
    if (!st.valid) { set_flag(flags, 1); return; }
    double dTp = 0.0, ratio = 0.0;
#pragma unroll
    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                double w = (double)(st.w[0][ox] * st.w[1][oy] * st.w[2][oz]);
                int64_t node = node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, R);
                dTp += w * __ldg(n_dT + node);
                double wn = __ldg(n_water + node);
                if (wn > 0.0) ratio += w * __ldg(n_dW + node) / wn;
            }
    double Tn = T_old[i] + dTp;
    double Wn = W_old[i] * (1.0 + ratio);
    double d = dry[i];
    T_new[i] = Tn;
    T_mat[i] = (float)Tn;
    W_new[i] = Wn;
    loss_new[i] = loss_old[i] + (double)dt * p_loss[i];
    exch_new[i] = exch_old[i] + (double)dt * p_heat[i];
    mass_new[i] = (float)(d + Wn);
    dens_new[i] = (float)((d + Wn) / (double)V0[i]);
    sat_new[i] = Wn / ((double)rho_w * (double)V0[i] * (double)det3(load_m3(Fp, i, pitch)));
}

// --------------------------------------------- thermal_water.py:232-260
__global__ void k_local_gas(int64_t n, int64_t pitch, const double* __restrict__ old_moles,
                            const double* __restrict__ T_old, const double* __restrict__ T_new,
                            double* __restrict__ new_moles, double* __restrict__ pressures,
                            const float* __restrict__ Fp, const float* __restrict__ por,
                            const float* __restrict__ parameter, int per_particle, float density, float peak,
                            float width, float dt, int produce) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = old_moles[i];
    double Tn = T_new[i];
    if (produce) {
        double Tm = 0.5 * (T_old[i] + Tn);
        double z = (Tm - (double)peak) / (double)width;
        m += (double)(dt * density) * (double)parameter[per_particle ? i : 0] * exp(-(z * z));
    }
    new_moles[i] = m;
    float ni = por[i];
    if (ni > 0.0f) pressures[i] = gas_pressure(m, (float)Tn, det3(load_m3(Fp, i, pitch)), ni);
}

__global__ void k_water_stress(int64_t n, int64_t pitch, const float* __restrict__ Fp, const double* __restrict__ sat,
                               const float* __restrict__ tau_old, float* __restrict__ tau_new, float s0, float k) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float iso = det3(load_m3(Fp, i, pitch)) * k * ((float)sat[i] - s0);
    M3 t = load_m3(tau_old, i, pitch);
#pragma unroll
    for (int e = 0; e < 9; ++e) t.m[e] -= (e % 4) == 0 ? iso : iso * 0.0f;
    store_m3(tau_new, i, pitch, t);
}

__global__ void k_saturations(int64_t n, int64_t pitch, const double* __restrict__ W, const float* __restrict__ V0,
                              const float* __restrict__ Fp, double* __restrict__ sat, float rho_w) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    sat[i] = W[i] / ((double)rho_w * (double)V0[i] * (double)det3(load_m3(Fp, i, pitch)));
}

// --------------------------------------------------- quasistatic.py:11-21
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float value) {
    // Non-negative floats order like their int bit patterns.
    if (value >= 0.0f) atomicMax(reinterpret_cast<int*>(addr), __float_as_int(value));
}

__global__ void k_settling_metrics(int64_t n, int64_t pitch, const float* __restrict__ v,
                                   const float* __restrict__ Cm, const float* __restrict__ Fo,
                                   const float* __restrict__ Fn, float* metrics, float dt) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    M3 a = load_m3(Cm, i, pitch), po = load_m3(Fo, i, pitch), pn = load_m3(Fn, i, pitch);
    V3 u = load_v3(v, i, pitch);
    float sym2 = 0, ch2 = 0, n2 = 0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float s = 0.5f * (a.m[3 * r + c] + a.m[3 * c + r]);
            sym2 += s * s;
            float d = pn.m[3 * r + c] - po.m[3 * r + c];
            ch2 += d * d;
            n2 += po.m[3 * r + c] * po.m[3 * r + c];
        }
    atomic_max_nonneg(metrics + 0, sqrtf(u.v[0] * u.v[0] + u.v[1] * u.v[1] + u.v[2] * u.v[2]));
    atomic_max_nonneg(metrics + 1, sqrtf(sym2));
    atomic_max_nonneg(metrics + 2, sqrtf(ch2) / (dt * sqrtf(n2)));
}

// --------------------------------------------- porous_return.py:34-61 (device evaluation)
__global__ void k_solve_porosity(int64_t n, const float* __restrict__ q, const float* __restrict__ p,
                                 const float* __restrict__ d, const float* __restrict__ h,
                                 const float* __restrict__ e, const double* __restrict__ Vp, float n0,
                                 float* __restrict__ out, double* __restrict__ pred) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    float r = solve_porosity(q[i], p[i], d[i], h[i], e[i], Vp[i], n0);
    out[i] = r;
    pred[i] = porosity_prediction((double)r, q[i], p[i], d[i], h[i], e[i], Vp[i], n0);
}

__global__ void k_porosity_coefficient(int64_t n, const float* __restrict__ por, float* __restrict__ out) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = porosity_coefficient(por[i]);
}

DingParamsDev to_dev(const BkDingParams& p) {
    DingParamsDev d;
    d.coupled_porosity = p.coupled_porosity;
    d.temperature_enabled = p.temperature_enabled;
    d.mu = p.shear_modulus; d.lam = p.lame_lambda; d.yield_stress = p.yield_stress;
    d.initial_porosity = p.initial_porosity; d.dt = p.time_step;
    for (int k = 0; k < 4; ++k) {
        d.knots[k] = p.temperature_knots[k];
        d.yield_factors[k] = p.yield_factors[k];
        d.viscosity_factors[k] = p.viscosity_factors[k];
    }
    return d;
}

bool bad_counts(int64_t n, int64_t pitch) { return n < 0 || pitch < n || n > (int64_t)INT32_MAX * 64; }

}  // namespace

// ===================================================================== C ABI
extern "C" {

int bk_version(void) { return 100; }

const char* bk_last_error(void) { return g_error; }

#define BK_REQUIRE(cond, msg) do { if (!(cond)) return fail(BK_ERR_ARGUMENT, msg); } while (0)
#define BK_EMPTY_OK(n) do { if ((n) == 0) return BK_OK; } while (0)

int bk_particle_to_grid(int64_t n, int64_t pitch, const float* x, const float* v, const float* C, const float* tau,
                        const float* mass, const float* V0, float* node_pm, const float* origin, float spacing,
                        int32_t resolution, float time_step, int32_t* flags, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_particle_to_grid: bad particle count/pitch");
    BK_REQUIRE(resolution > 0 && spacing > 0.0f && origin, "bk_particle_to_grid: bad grid");
    BK_EMPTY_OK(n);
    BK_REQUIRE(x && v && C && tau && mass && V0 && node_pm && flags, "bk_particle_to_grid: null pointer");
    BK_REQUIRE(((uintptr_t)node_pm & 15) == 0, "bk_particle_to_grid: node_pm must be 16-byte aligned");
    k_particle_to_grid<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, x, v, C, tau, mass, V0,
                                                               reinterpret_cast<float4*>(node_pm),
                                                               origin_of(origin), spacing, resolution, time_step,
                                                               flags);
    return check_launch("bk_particle_to_grid");
}

int bk_update_grid(int32_t resolution, const float* node_pm, float* node_v, int32_t boundary_cells,
                   const float* gravity, float time_step, void* stream) {
    BK_REQUIRE(resolution > 0 && node_pm && node_v && gravity, "bk_update_grid: bad arguments");
    BK_REQUIRE((((uintptr_t)node_pm | (uintptr_t)node_v) & 15) == 0, "bk_update_grid: node arrays must be 16-byte aligned");
    int64_t nn = (int64_t)resolution * resolution * resolution;
    k_update_grid<<<blocks_for(nn), kBlock, 0, S(stream)>>>(resolution, reinterpret_cast<const float4*>(node_pm),
                                                           reinterpret_cast<float4*>(node_v), boundary_cells,
                                                           gravity[0], gravity[1], gravity[2], time_step);
    return check_launch("bk_update_grid");
}

int bk_grid_to_particle(int64_t n, int64_t pitch, const float* x_in, const float* F_in, const float* node_v,
                        float* x_out, float* v_out, float* C_out, float* F_out, const float* origin, float spacing,
                        int32_t resolution, float time_step, int32_t* flags, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_grid_to_particle: bad particle count/pitch");
    BK_REQUIRE(resolution > 0 && spacing > 0.0f && origin, "bk_grid_to_particle: bad grid");
    BK_EMPTY_OK(n);
    BK_REQUIRE(x_in && F_in && node_v && x_out && v_out && C_out && F_out && flags, "bk_grid_to_particle: null pointer");
    BK_REQUIRE(((uintptr_t)node_v & 15) == 0, "bk_grid_to_particle: node_v must be 16-byte aligned");
    k_grid_to_particle<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, x_in, F_in,
                                                               reinterpret_cast<const float4*>(node_v), x_out,
                                                               v_out, C_out, F_out, origin_of(origin), spacing,
                                                               resolution, time_step, flags);
    return check_launch("bk_grid_to_particle");
}

int bk_compute_elastic_stress(int64_t n, int64_t pitch, const float* F, float* tau, float mu, float lam,
                              int32_t* flags, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_compute_elastic_stress: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(F && tau && flags, "bk_compute_elastic_stress: null pointer");
    k_elastic_stress<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, F, tau, mu, lam, flags);
    return check_launch("bk_compute_elastic_stress");
}

int bk_update_ding(int64_t n, int64_t pitch, const float* Fe_old, const float* porosity_old, const int32_t* gelled_old,
                   const float* F_total, const float* C_new, float* Fe_new, float* Fp_new, float* tau_new,
                   float* residuals, float* porosity_new, float* temperature_out, int32_t* gelled_new,
                   float* yield_out, float* viscosity_out, const float* viscosity_parameter, int32_t* flags,
                   float* porosity_residuals, const BkDingParams* params, const float* temperature_local,
                   void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_update_ding: bad count/pitch");
    BK_REQUIRE(params != nullptr, "bk_update_ding: null params");
    BK_EMPTY_OK(n);
    BK_REQUIRE(Fe_old && porosity_old && gelled_old && F_total && C_new && Fe_new && Fp_new && tau_new && residuals &&
               porosity_new && temperature_out && gelled_new && yield_out && viscosity_out && viscosity_parameter &&
               flags && porosity_residuals && temperature_local, "bk_update_ding: null pointer");
    k_update_ding<<<blocks_for(n, 128), 128, 0, S(stream)>>>(
        n, pitch, Fe_old, porosity_old, gelled_old, F_total, C_new, Fe_new, Fp_new, tau_new, residuals, porosity_new,
        temperature_out, gelled_new, yield_out, viscosity_out, viscosity_parameter, flags, porosity_residuals,
        to_dev(*params), temperature_local);
    return check_launch("bk_update_ding");
}

int bk_combine_gas_stress(int64_t n, int64_t pitch, const float* tau_solid, const float* F, const float* porosity,
                          const double* moles, const float* temperature, float* tau_total, int32_t* flags,
                          float ambient_pressure, float initial_porosity, const float* density, float elastic_modulus,
                          float time_step, float spacing, float cfl_limit, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_combine_gas_stress: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(tau_solid && F && porosity && moles && temperature && tau_total && flags && density,
               "bk_combine_gas_stress: null pointer");
    k_combine_gas_stress<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, tau_solid, F, porosity, moles,
                                                                 temperature, tau_total, flags, ambient_pressure,
                                                                 initial_porosity, density, elastic_modulus,
                                                                 time_step, spacing, cfl_limit);
    return check_launch("bk_combine_gas_stress");
}

int bk_refresh_gas(int64_t n, int64_t pitch, const double* old_moles, double* new_moles, const float* F,
                   const float* porosity, double* pressures, const float* temperature, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_refresh_gas: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(old_moles && new_moles && F && porosity && pressures && temperature, "bk_refresh_gas: null pointer");
    k_refresh_gas<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, old_moles, new_moles, F, porosity, pressures,
                                                          temperature);
    return check_launch("bk_refresh_gas");
}

int bk_reconstruct_mesh_vertices(int64_t vertex_count, int64_t pitch, const float* x, const float* F,
                                 int64_t vertex_pitch, const float* reference_vertices, const int32_t* offsets,
                                 const int32_t* particles, const float* weights, int64_t binding_pitch,
                                 const float* reference_offsets, float* out_vertices, void* stream) {
    BK_REQUIRE(vertex_count >= 0 && vertex_pitch >= vertex_count && pitch >= 0, "bk_reconstruct_mesh_vertices: bad sizes");
    BK_EMPTY_OK(vertex_count);
    BK_REQUIRE(x && F && reference_vertices && offsets && particles && weights && reference_offsets && out_vertices,
               "bk_reconstruct_mesh_vertices: null pointer");
    BK_REQUIRE(vertex_count <= INT32_MAX, "bk_reconstruct_mesh_vertices: too many vertices");
    const unsigned nv = (unsigned)vertex_count;
    // binding_pitch bounds the total bindings: the launch-size hint of vertex_block_threads
    switch (vertex_block_threads(vertex_count, binding_pitch)) {
        case 256:
            k_reconstruct_vertices<256><<<nv, 256, 0, S(stream)>>>(pitch, x, F, vertex_pitch, reference_vertices, offsets,
                                                                  particles, weights, binding_pitch, reference_offsets,
                                                                  out_vertices);
            break;
        case 128:
            k_reconstruct_vertices<128><<<nv, 128, 0, S(stream)>>>(pitch, x, F, vertex_pitch, reference_vertices, offsets,
                                                                  particles, weights, binding_pitch, reference_offsets,
                                                                  out_vertices);
            break;
        default:
            k_reconstruct_vertices<32><<<nv, 32, 0, S(stream)>>>(pitch, x, F, vertex_pitch, reference_vertices, offsets,
                                                                particles, weights, binding_pitch, reference_offsets,
                                                                out_vertices);
            break;
    }
    return check_launch("bk_reconstruct_mesh_vertices");
}

int bk_surface_areas(int64_t face_count, int64_t vertex_pitch, const float* vertices, const int32_t* faces,
                     const int32_t* owners, double* exposed, double* contact, float floor_height,
                     float contact_distance, void* stream) {
    BK_REQUIRE(face_count >= 0, "bk_surface_areas: bad count");
    BK_EMPTY_OK(face_count);
    BK_REQUIRE(vertices && faces && owners && exposed && contact, "bk_surface_areas: null pointer");
    k_surface_areas<<<blocks_for(face_count), kBlock, 0, S(stream)>>>(face_count, vertex_pitch, vertices, faces,
                                                                     owners, exposed, contact, floor_height,
                                                                     contact_distance);
    return check_launch("bk_surface_areas");
}

int bk_scalar_to_grid(int64_t n, int64_t pitch, const float* x, const float* F, const float* V0,
                      const double* capacities, const double* temperatures, const double* water,
                      const double* exposed, const double* contact, const float* heat_parameter,
                      const BkScalarParams* params, double* const* node_fields, double* particle_heat,
                      double* particle_loss, int32_t* flags, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_scalar_to_grid: bad count/pitch");
    BK_REQUIRE(params && node_fields, "bk_scalar_to_grid: null params");
    BK_EMPTY_OK(n);
    BK_REQUIRE(x && F && V0 && capacities && temperatures && water && exposed && contact && heat_parameter &&
               particle_heat && particle_loss && flags, "bk_scalar_to_grid: null pointer");
    ScalarParamsDev P;
    P.oven = params->oven_temperature; P.tray = params->tray_temperature; P.tray_transfer = params->tray_transfer;
    P.surface_loss = params->surface_loss; P.water_density = params->water_density; P.latent = params->latent_heat;
    P.water_enabled = params->water_enabled;
    for (int a = 0; a < 3; ++a) P.origin[a] = params->origin[a];
    P.dx = params->spacing; P.R = params->resolution;
    NodeFields nf;
    for (int k = 0; k < 7; ++k) {
        BK_REQUIRE(node_fields[k] != nullptr, "bk_scalar_to_grid: null node field");
        nf.f[k] = node_fields[k];
    }
    k_scalar_to_grid<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, x, F, V0, capacities, temperatures, water,
                                                             exposed, contact, heat_parameter, P, nf, particle_heat,
                                                             particle_loss, flags);
    return check_launch("bk_scalar_to_grid");
}

int bk_grid_fields(int64_t node_count, const double* volumes, const double* capacities, const double* energy,
                   const double* water, double* temperatures, double* saturations, float water_density,
                   void* stream) {
    BK_REQUIRE(node_count >= 0, "bk_grid_fields: bad count");
    BK_EMPTY_OK(node_count);
    BK_REQUIRE(volumes && capacities && energy && water && temperatures && saturations, "bk_grid_fields: null pointer");
    k_grid_fields<<<blocks_for(node_count), kBlock, 0, S(stream)>>>(node_count, volumes, capacities, energy, water,
                                                                   temperatures, saturations, water_density);
    return check_launch("bk_grid_fields");
}

int bk_diffuse_grid(int64_t node_count, const double* volumes, const double* capacities, const double* temperatures,
                    const double* saturations, const double* water, const double* boundary_heat,
                    const double* boundary_loss, const double* boundary_exchange, double* temperature_changes,
                    double* water_changes, int32_t* errors, float conductivity, float diffusivity,
                    float water_density, int32_t water_enabled, float spacing, int32_t resolution, float time_step,
                    void* stream) {
    BK_REQUIRE(resolution > 0 && node_count == (int64_t)resolution * resolution * resolution,
               "bk_diffuse_grid: node_count must be resolution^3");
    BK_REQUIRE(volumes && capacities && temperatures && saturations && water && boundary_heat && boundary_loss &&
               boundary_exchange && temperature_changes && water_changes && errors, "bk_diffuse_grid: null pointer");
    k_diffuse_grid<<<blocks_for(node_count), kBlock, 0, S(stream)>>>(
        node_count, volumes, capacities, temperatures, saturations, water, boundary_heat, boundary_loss,
        boundary_exchange, temperature_changes, water_changes, errors, conductivity, diffusivity, water_density,
        water_enabled, spacing, resolution, time_step);
    return check_launch("bk_diffuse_grid");
}

int bk_scalar_to_particles(int64_t n, int64_t pitch, const float* x, const double* T_old, const double* W_old,
                           const double* loss_old, const double* exchange_old, const double* dry_masses,
                           const float* V0, const float* F, const double* node_water, const double* node_dT,
                           const double* node_dW, const double* particle_heat, const double* particle_loss,
                           double* T_new, float* T_material, double* W_new, double* loss_new, double* exchange_new,
                           float* mass_new, float* density_new, double* saturation_new, float water_density,
                           const float* origin, float spacing, int32_t resolution, float time_step, int32_t* flags,
                           void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_scalar_to_particles: bad count/pitch");
    BK_REQUIRE(resolution > 0 && spacing > 0.0f && origin, "bk_scalar_to_particles: bad grid");
    BK_EMPTY_OK(n);
    BK_REQUIRE(x && T_old && W_old && loss_old && exchange_old && dry_masses && V0 && F && node_water && node_dT &&
               node_dW && particle_heat && particle_loss && T_new && T_material && W_new && loss_new &&
               exchange_new && mass_new && density_new && saturation_new && flags,
               "bk_scalar_to_particles: null pointer");
    k_scalar_to_particles<<<blocks_for(n), kBlock, 0, S(stream)>>>(
        n, pitch, x, T_old, W_old, loss_old, exchange_old, dry_masses, V0, F, node_water, node_dT, node_dW,
        particle_heat, particle_loss, T_new, T_material, W_new, loss_new, exchange_new, mass_new, density_new,
        saturation_new, water_density, origin_of(origin), spacing, resolution, time_step, flags);
    return check_launch("bk_scalar_to_particles");
}

int bk_local_gas(int64_t n, int64_t pitch, const double* old_moles, const double* T_old, const double* T_new,
                 double* new_moles, double* pressures, const float* F, const float* porosity, const float* parameter,
                 int32_t per_particle, float density, float peak, float width, float time_step, int32_t produce,
                 void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_local_gas: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(old_moles && T_old && T_new && new_moles && pressures && F && porosity && parameter,
               "bk_local_gas: null pointer");
    k_local_gas<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, old_moles, T_old, T_new, new_moles, pressures, F,
                                                        porosity, parameter, per_particle, density, peak, width,
                                                        time_step, produce);
    return check_launch("bk_local_gas");
}

int bk_water_stress(int64_t n, int64_t pitch, const float* F, const double* saturations, const float* tau_old,
                    float* tau_new, float initial_saturation, float stiffness, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_water_stress: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(F && saturations && tau_old && tau_new, "bk_water_stress: null pointer");
    k_water_stress<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, F, saturations, tau_old, tau_new,
                                                           initial_saturation, stiffness);
    return check_launch("bk_water_stress");
}

int bk_saturations(int64_t n, int64_t pitch, const double* water, const float* V0, const float* F,
                   double* saturations, float density, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_saturations: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(water && V0 && F && saturations, "bk_saturations: null pointer");
    k_saturations<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, water, V0, F, saturations, density);
    return check_launch("bk_saturations");
}

int bk_settling_metrics(int64_t n, int64_t pitch, const float* v, const float* C, const float* Fp_old,
                        const float* Fp_new, float* metrics, float time_step, void* stream) {
    BK_REQUIRE(!bad_counts(n, pitch), "bk_settling_metrics: bad count/pitch");
    BK_EMPTY_OK(n);
    BK_REQUIRE(v && C && Fp_old && Fp_new && metrics, "bk_settling_metrics: null pointer");
    k_settling_metrics<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, pitch, v, C, Fp_old, Fp_new, metrics, time_step);
    return check_launch("bk_settling_metrics");
}

int bk_solve_porosity(int64_t n, const float* q, const float* p, const float* dev_factor, const float* mean_scale,
                      const float* exponent, const double* plastic_volume, float initial_porosity, float* porosity,
                      double* prediction, void* stream) {
    BK_REQUIRE(n >= 0, "bk_solve_porosity: bad count");
    BK_EMPTY_OK(n);
    BK_REQUIRE(q && p && dev_factor && mean_scale && exponent && plastic_volume && porosity && prediction,
               "bk_solve_porosity: null pointer");
    k_solve_porosity<<<blocks_for(n, 128), 128, 0, S(stream)>>>(n, q, p, dev_factor, mean_scale, exponent,
                                                               plastic_volume, initial_porosity, porosity,
                                                               prediction);
    return check_launch("bk_solve_porosity");
}

int bk_porosity_coefficient(int64_t n, const float* porosity, float* coefficient, void* stream) {
    BK_REQUIRE(n >= 0, "bk_porosity_coefficient: bad count");
    BK_EMPTY_OK(n);
    BK_REQUIRE(porosity && coefficient, "bk_porosity_coefficient: null pointer");
    k_porosity_coefficient<<<blocks_for(n), kBlock, 0, S(stream)>>>(n, porosity, coefficient);
    return check_launch("bk_porosity_coefficient");
}

}  // extern "C"
