// Adjoint of the thermal-water transport part of one substep, the companion of
// bk_substep_adjoint: the forward transport phase (physics/thermal_water.py:77-190 -- surface
// areas, scalar P2G, diffusion) and the scalar G2P with its water stress and mass
// (thermal_water.py:193-229, 248-253) and, in gas mode, its local gas source and gas-pressure
// stress (thermal_water.py:232-245, physics/materials/gas.py:16-35) reversed, given the substep's
// grid with its transport fields
// kept (BkSubstepParams.keep_transport_fields) and the adjoints the mechanics adjoint produced for
// the stress, particle mass and material temperature that P2G and the return map used.
//
// Order, all per substep:
//   prepare          T_mat = T + sum w dT, mass = dry + W', stress tau + J (p_amb - p) I
//                    - J c (s - s0) I: the inputs bk_substep_adjoint needs (call before it)
//   scalar_chain     dL/d(T', W', N', T_mat, mass, stress) -> dL/d(T, W, N, n, F, x, alpha) and
//                    the node adjoints of (dT, dW/W)
//   diffuse          node gather: dL/d(dT, dW/W) -> dL/d(volume, capacity, energy, water, heat, loss)
//   scatter          particle gather of the node-field adjoints -> dL/d(F, T, W, x)
//   owners           surface heat/loss of face-owning particles -> dL/d(T, W, F, x, h) and the
//                    face-vertex adjoints
//   vertices         mesh-vertex adjoints -> dL/d(x, F) of the bound particles
//   clear            zero the kept fields and every node scratch array over the active box
// Node scratch arrays start at zero and are left at zero. Discrete switches (tray contact test,
// nodes without capacity, the stability flags) carry no gradient.
#include <climits>
#include <cstdio>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"

using namespace bk;

namespace {

constexpr int kThreads = 128;

// The forward substep's transport node fields (volume, capacity, energy, water, heat, loss,
// exchange) and the node adjoint scratch arrays.
struct BkGridFields {
    double* fields[7];
    double* field_bar[6];
    double2* dTr_bar;
};

struct TParams {
    int64_t n, pitch;
    int R;
    float origin[3], dx, dt;
    double rho_w, s0, c_water, kc, kw, cell;
    int water_enabled;
    double oven, tray, tray_transfer, surface_loss, latent;
    double contact_limit;  // floor height + contact distance, summed in float as the forward does
    int gas, settling;
    double ambient, peak, width, source_scale;  // gas: ambient pressure, source peak/width, dt * density
};

__device__ __forceinline__ float qgrad(float l, int o) {
    if (o == 0) return -(1.5f - l);
    if (o == 1) return -2.f * (l - 1.f);
    return l - 0.5f;
}

__device__ __forceinline__ void node_offset(int j, int& ox, int& oy, int& oz) {
    ox = j / 9;
    oy = (j / 3) % 3;
    oz = j - 9 * ox - 3 * oy;
}

// Weight of stencil node j and its gradient with respect to the particle position.
__device__ __forceinline__ float weight_and_grad(const Stencil& st, int ox, int oy, int oz, float inv_dx, float* dw) {
    const float wx = st.w[0][ox], wy = st.w[1][oy], wz = st.w[2][oz];
    dw[0] = qgrad(st.l[0], ox) * inv_dx * wy * wz;
    dw[1] = qgrad(st.l[1], oy) * inv_dx * wx * wz;
    dw[2] = qgrad(st.l[2], oz) * inv_dx * wx * wy;
    return wx * wy * wz;
}

__device__ __forceinline__ void add_det_grad(float* Fb, int64_t i, int64_t pitch, const M3& F, float scale) {
    // d det(F) / dF = det(F) F^-T; adds scale * det(F) F^-T
    const M3 inv = inverse3(F);
    const float J = det3(F);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Fb[(3 * r + c) * pitch + i] += scale * J * inv.m[3 * c + r];
}

// Gas content after this substep's local source (thermal_water.py:238-245):
// N' = N + dt rho alpha exp(-z^2), z = ((T + T')/2 - T_peak) / width; no source while settling.
// `ez`, `z` (may be NULL) return exp(-z^2) and z.
__device__ __forceinline__ double source_moles(const TParams& P, const BkState& in, const BkConstants& cst, int64_t i,
                                               double T, double Tn, double* ez, double* z) {
    double N = in.gas_moles[i];
    if (!P.settling) {
        const double zz = (0.5 * (T + Tn) - P.peak) / P.width;
        const double e = exp(-(zz * zz));
        N += P.source_scale * (double)cst.gas_rate[cst.gas_rate_per_particle ? i : 0] * e;
        if (ez) *ez = e;
        if (z) *z = zz;
    }
    return N;
}

// ------------------------------------------------------------------ prepare
__global__ void k_tadj_prepare(TParams P, BkState in, BkConstants cst, const double2* __restrict__ dTr,
                               float* __restrict__ T_mat, float* __restrict__ mass, float* __restrict__ tau_eff) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int64_t pitch = P.pitch;
    Stencil st = make_stencil(load_v3(in.x, i, pitch), P.origin, P.dx, P.R);
    if (!st.valid) return;
    double dTp = 0.0, ratio = 0.0;
#pragma unroll
    for (int j = 0; j < 27; ++j) {
        int ox, oy, oz;
        node_offset(j, ox, oy, oz);
        const double w = (double)(st.w[0][ox] * st.w[1][oy] * st.w[2][oz]);
        const double2 d = dTr[node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R)];
        dTp += w * d.x;
        ratio += w * d.y;
    }
    const double T = in.temperature[i];
    const double Tn = T + dTp, Wn = in.water[i] * (1.0 + ratio);
    T_mat[i] = (float)Tn;
    mass[i] = (float)(cst.dry_mass[i] + Wn);
    const M3 F = load_m3(in.F, i, pitch);
    const float J = det3(F);
    M3 tau = load_m3(in.tau, i, pitch);
    if (P.gas) {
        const float n = in.porosity[i];
        if (n > 0.0f && n < 1.0f && isfinite(n) && J > 0.0f) {
            const float p = (float)gas_pressure(source_moles(P, in, cst, i, T, Tn, nullptr, nullptr), (float)Tn, J, n);
            const float iso = J * ((float)P.ambient - p);
#pragma unroll
            for (int e = 0; e < 9; ++e) tau.m[e] += (e % 4) == 0 ? iso : 0.0f;
        }
    }
    const double sat = Wn / (P.rho_w * (double)cst.volume[i] * (double)J);
    const float iso = J * (float)P.c_water * ((float)sat - (float)P.s0);
#pragma unroll
    for (int e = 0; e < 9; ++e) tau.m[e] -= (e % 4) == 0 ? iso : 0.0f;
    store_m3(tau_eff, i, pitch, tau);
}

// ------------------------------------------------------------- scalar chain
// Node adjoints of (dT, dW/W) are scattered like the forward's scalar P2G: a block stages the node
// box its particles touch in shared memory (when it fits kTileNodes), and within a warp each run
// of particles with the same stencil base is summed by 27 lanes, one node each, before one atomic
// per node.
constexpr int kTileNodes = 512;

struct ScalarSmem {
    float w[kThreads][9];
    double val[kThreads][2];
    double tile[2][kTileNodes];
    int box[6];
};

__device__ __forceinline__ long long pack_base(const int* b) {
    return ((long long)b[0] << 42) | ((long long)b[1] << 21) | (long long)b[2];
}

__global__ void __launch_bounds__(kThreads) k_tadj_scalar(TParams P, BkState in, BkConstants cst,
                                                        const double2* __restrict__ dTr, BkAdjointTransport a,
                                                        const BkAdjointState adj, double2* __restrict__ dTr_bar) {
    __shared__ ScalarSmem sm;
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + tid;
    const int64_t pitch = P.pitch;
    double rate_b = 0.0;  // dL/d(gas source rate) through this particle
    double Tnb = 0.0, ratiob = 0.0;
    Stencil st;
    st.valid = false;
    st.b[0] = st.b[1] = st.b[2] = 0;
    if (i < P.n) st = make_stencil(load_v3(in.x, i, pitch), P.origin, P.dx, P.R);
    const bool valid = i < P.n && st.valid;
    if (i < P.n && !st.valid) {
        a.temperature_in[i] = 0.0;
        a.water_in[i] = 0.0;
        if (P.gas) a.gas_moles_in[i] = 0.0;
    } else if (valid) {
        // one pass over the stencil: T' and W' need sum w (dT, r); the weight gradients of x need
        // sum grad w (dT, r), which do not depend on the adjoints
        double dTp = 0.0, ratio = 0.0;
        float gT[3] = {0.f, 0.f, 0.f}, gr[3] = {0.f, 0.f, 0.f};
        const float inv_dx = 1.f / P.dx;
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            int ox, oy, oz;
            node_offset(j, ox, oy, oz);
            float dw[3];
            const double w = (double)weight_and_grad(st, ox, oy, oz, inv_dx, dw);
            const double2 d = dTr[node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R)];
            dTp += w * d.x;
            ratio += w * d.y;
            const float fx = (float)d.x, fy = (float)d.y;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                gT[c] += dw[c] * fx;
                gr[c] += dw[c] * fy;
            }
        }
        const double T = in.temperature[i], Tn = T + dTp;
        const double W = in.water[i];
        const double Wn = W * (1.0 + ratio);
        const M3 F = load_m3(in.F, i, pitch);
        const float Jf = det3(F);
        const double J = (double)Jf;
        const double V0 = (double)cst.volume[i];
        const double sat = Wn / (P.rho_w * V0 * J);
        // adjoints arriving at T', W', T_mat, mass and the P2G stress
        Tnb = a.temperature_out[i] + (double)adj.temperature[i];
        double Wnb = a.water_out[i] + (double)adj.mass[i];
        const double trace = (double)adj.tau[i] + (double)adj.tau[4 * pitch + i] + (double)adj.tau[8 * pitch + i];
        // stress -= iso I, iso = J c (s - s0)
        const double isob = -trace;
        double Jb = isob * P.c_water * (sat - P.s0);
        const double satb = isob * J * P.c_water;
        Wnb += satb / (P.rho_w * V0 * J);
        Jb -= satb * sat / J;
        double Tb_direct = 0.0;  // through the source's mean temperature, besides T'
        if (P.gas) {
            double ez = 0.0, z = 0.0;
            const double Np = source_moles(P, in, cst, i, T, Tn, &ez, &z);
            double Npb = a.gas_moles_out[i];
            const float n = in.porosity[i];
            if (n > 0.0f && n < 1.0f && isfinite(n) && Jf > 0.0f) {
                // stress += J (p_amb - p) I, p = N' R T_mat / (J n) (gas.py:11-13, 27-29)
                const float Tm = (float)Tn;
                const double pg = (double)(float)gas_pressure(Np, Tm, Jf, n);
                Jb += trace * (P.ambient - pg);
                const double pb = -trace * J;
                Npb += pb * kGasConstant * (double)Tm / (J * (double)n);
                Tnb += pb * pg / (double)Tm;
                Jb -= pb * pg / J;
                adj.porosity[i] += (float)(-pb * pg / (double)n);
            }
            a.gas_moles_in[i] = Npb;
            if (!P.settling) {
                const double rate = (double)cst.gas_rate[cst.gas_rate_per_particle ? i : 0];
                rate_b = Npb * P.source_scale * ez;
                const double zb = Npb * P.source_scale * rate * ez * (-2.0 * z);
                Tnb += zb * 0.5 / P.width;
                Tb_direct = zb * 0.5 / P.width;
            }
        }
        // W' = W (1 + sum w r), T' = T + sum w dT
        ratiob = Wnb * W;
        a.water_in[i] = Wnb * (1.0 + ratio);
        a.temperature_in[i] = Tnb + Tb_direct;
        // weight gradients: x_bar += sum_j grad w_j (dT_j T'_bar + r_j ratio_bar)
        const float tb = (float)Tnb, rb = (float)ratiob;
#pragma unroll
        for (int c = 0; c < 3; ++c) adj.x[c * pitch + i] += gT[c] * tb + gr[c] * rb;
        add_det_grad(adj.F, i, pitch, F, (float)Jb);
    }
    // ---- scatter w (T'_bar, ratio_bar) into the node adjoints
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
#pragma unroll
        for (int o = 0; o < 3; ++o) sm.w[tid][3 * ax + o] = valid ? st.w[ax][o] : 0.f;
    sm.val[tid][0] = Tnb;
    sm.val[tid][1] = ratiob;
    if (tid < 6) sm.box[tid] = tid < 3 ? INT_MAX : INT_MIN;
    __syncthreads();
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int lo = __reduce_min_sync(0xffffffffu, valid ? st.b[ax] : INT_MAX);
        const int hi = __reduce_max_sync(0xffffffffu, valid ? st.b[ax] + 2 : INT_MIN);
        if (lane == 0 && lo != INT_MAX) {
            atomicMin(&sm.box[ax], lo);
            atomicMax(&sm.box[3 + ax], hi);
        }
    }
    __syncthreads();
    int lo[3] = {0, 0, 0}, ext[3] = {1, 1, 1};
    int count = 0;
    bool tiled = false;
    if (sm.box[0] != INT_MAX) {
        long long c = 1;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            lo[ax] = sm.box[ax];
            ext[ax] = sm.box[3 + ax] - sm.box[ax] + 1;
            c *= ext[ax];
        }
        tiled = c <= kTileNodes;
        count = tiled ? (int)c : 0;
    }
    for (int t = tid; t < count; t += kThreads) sm.tile[0][t] = sm.tile[1][t] = 0.0;
    __syncthreads();
    const long long key = valid ? pack_base(st.b) : -1;
    const long long prev = __shfl_up_sync(0xffffffffu, key, 1);
    unsigned starts = __ballot_sync(0xffffffffu, valid && (lane == 0 || prev != key));
    const int warp_base = tid & ~31;
    int ox, oy, oz;
    node_offset(lane < 27 ? lane : 0, ox, oy, oz);
    while (starts) {
        const int s0 = __ffs(starts) - 1;
        starts &= starts - 1;
        const int e = starts ? __ffs(starts) - 1 : 32;
        const int b0 = __shfl_sync(0xffffffffu, st.b[0], s0), b1 = __shfl_sync(0xffffffffu, st.b[1], s0),
                  b2 = __shfl_sync(0xffffffffu, st.b[2], s0);
        if (lane < 27) {
            double acc0 = 0.0, acc1 = 0.0;
            for (int k = warp_base + s0; k < warp_base + e; ++k) {
                const double w = (double)(sm.w[k][ox] * sm.w[k][3 + oy] * sm.w[k][6 + oz]);
                acc0 += w * sm.val[k][0];
                acc1 += w * sm.val[k][1];
            }
            if (tiled) {
                const int t = ((b0 + ox - lo[0]) * ext[1] + (b1 + oy - lo[1])) * ext[2] + (b2 + oz - lo[2]);
                atomicAdd(&sm.tile[0][t], acc0);
                atomicAdd(&sm.tile[1][t], acc1);
            } else {
                double2* d = dTr_bar + node_index(b0 + ox, b1 + oy, b2 + oz, P.R);
                atomicAdd(&d->x, acc0);
                atomicAdd(&d->y, acc1);
            }
        }
    }
    __syncthreads();
    for (int t = tid; t < count; t += kThreads) {
        const double v0 = sm.tile[0][t], v1 = sm.tile[1][t];
        if (v0 == 0.0 && v1 == 0.0) continue;
        const int z = t % ext[2], y = (t / ext[2]) % ext[1], x = t / (ext[2] * ext[1]);
        double2* d = dTr_bar + node_index(lo[0] + x, lo[1] + y, lo[2] + z, P.R);
        atomicAdd(&d->x, v0);
        atomicAdd(&d->y, v1);
    }
    if (P.gas && a.gas_rate) {
        if (cst.gas_rate_per_particle) {
            if (i < P.n) a.gas_rate[i] += rate_b;
        } else {
            // one shared rate: a warp sum, then one atomic per warp
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) rate_b += __shfl_xor_sync(0xffffffffu, rate_b, o);
            if (lane == 0 && rate_b != 0.0) atomicAdd(a.gas_rate, rate_b);
        }
    }
}

// ------------------------------------------------------------------ diffuse
// For node i with capacity: T_i = E_i / c_i, s_i = W_i / (rho_w v_i); heat rate
// H_i + sum_j kc fill_ij (T_j - T_i); water rate -Lo_i + sum_j mob_ij (s_j - s_i) with
// mob_ij = kw fill_ij (T_i + T_j)(s_i + s_j) / 4, fill_ij = 2 v_i v_j / ((v_i + v_j) cell);
// dT_i = dt heat_i / c_i, (dW/W)_i = dt water_i / W_i. Node i gathers the adjoints of its own rates
// and of its 6 neighbours' rates (which use its T, s, v), so no atomics are needed.
struct NodeVals {
    double v, c, T, s, W;
    bool live;
};

__device__ __forceinline__ NodeVals node_vals(const TParams& P, double* const* f, int64_t i) {
    NodeVals n;
    n.c = f[1][i];
    n.live = n.c > 0.0;
    n.v = f[0][i];
    n.W = f[3][i];
    n.T = n.live ? f[2][i] / n.c : 0.0;
    n.s = n.live ? n.W / (P.rho_w * n.v) : 0.0;
    return n;
}

__global__ void k_tadj_diffuse(TParams P, BkGridFields g, const int32_t* __restrict__ box) {
    int lo[3], ext[3];
    int64_t count = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int l = max(box[k], 0), h = min(box[3 + k], P.R - 1);
        if (l > h) return;
        lo[k] = l;
        ext[k] = h - l + 1;
        count *= ext[k];
    }
    const int R = P.R;
    const double dt = (double)P.dt;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        int c[3];
        c[2] = lo[2] + (int)(t % ext[2]);
        c[1] = lo[1] + (int)((t / ext[2]) % ext[1]);
        c[0] = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        const int64_t i = node_index(c[0], c[1], c[2], R);
        const NodeVals ni = node_vals(P, g.fields, i);
        double vb = 0.0, cb = 0.0, Eb = 0.0, Wb = 0.0, Hb = 0.0, Lb = 0.0, Tb = 0.0, sb = 0.0;
        if (ni.live) {
            const double2 ob = g.dTr_bar[i];
            // own outputs
            const double heat_b = ob.x * dt / ni.c;
            double heat_rate = g.fields[4][i], water_rate = -g.fields[5][i];
            // rates are needed for the c_i and W_i terms: recompute them below with the neighbours
            const double water_b = ni.W > 0.0 ? ob.y * dt / ni.W : 0.0;
            Hb = heat_b;
            Lb = -water_b;
#pragma unroll
            for (int axis = 0; axis < 3; ++axis)
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    int o[3] = {c[0], c[1], c[2]};
                    o[axis] += 2 * side - 1;
                    if (o[axis] < 0 || o[axis] >= R) continue;
                    const int64_t j = node_index(o[0], o[1], o[2], R);
                    const NodeVals nj = node_vals(P, g.fields, j);
                    if (!nj.live) continue;
                    const double sum = ni.v + nj.v;
                    const double fill = 2.0 * ni.v * nj.v / sum / P.cell;
                    const double dfill_i = 2.0 * nj.v * nj.v / (sum * sum) / P.cell;  // d fill / d v_i
                    const double hc = P.kc * fill;
                    heat_rate += hc * (nj.T - ni.T);
                    // the neighbour's heat-rate adjoint
                    const double2 jb = g.dTr_bar[j];
                    const double heat_bj = jb.x * dt / nj.c;
                    // own rate: hc (T_j - T_i); neighbour's rate: hc (T_i - T_j)
                    Tb += -heat_b * hc + heat_bj * hc;
                    vb += (heat_b * (nj.T - ni.T) + heat_bj * (ni.T - nj.T)) * P.kc * dfill_i;
                    if (P.water_enabled) {
                        const double water_bj = nj.W > 0.0 ? jb.y * dt / nj.W : 0.0;
                        const double q = P.kw * fill * 0.25;
                        const double mob = q * (ni.T + nj.T) * (ni.s + nj.s);
                        water_rate += mob * (nj.s - ni.s);
                        // own: mob (s_j - s_i); neighbour's: mob (s_i - s_j)
                        const double ds_own = nj.s - ni.s, ds_nb = ni.s - nj.s;
                        sb += water_b * (-mob + ds_own * q * (ni.T + nj.T)) + water_bj * (mob + ds_nb * q * (ni.T + nj.T));
                        Tb += (water_b * ds_own + water_bj * ds_nb) * q * (ni.s + nj.s);
                        vb += (water_b * ds_own + water_bj * ds_nb) * (mob / fill) * dfill_i;
                    }
                }
            // dT_i = dt heat_rate / c_i, ratio_i = dt water_rate / W_i
            cb -= ob.x * dt * heat_rate / (ni.c * ni.c);
            if (ni.W > 0.0) Wb -= ob.y * dt * water_rate / (ni.W * ni.W);
            // T_i = E_i / c_i, s_i = W_i / (rho_w v_i)
            Eb += Tb / ni.c;
            cb -= Tb * ni.T / ni.c;
            Wb += sb / (P.rho_w * ni.v);
            vb -= sb * ni.s / ni.v;
        }
        g.field_bar[0][i] = vb;
        g.field_bar[1][i] = cb;
        g.field_bar[2][i] = Eb;
        g.field_bar[3][i] = Wb;
        g.field_bar[4][i] = Hb;
        g.field_bar[5][i] = Lb;
    }
}

// ------------------------------------------------------------------ scatter
// Node fields (volume V0 det F, capacity, capacity T, W) += w (...) for every particle: the
// reverse of that scatter is a 27-node gather of the four field adjoints. The block first stages
// the adjoints of its particles' node box in shared memory (when the box fits kScatterTile nodes),
// so that the gathers read shared memory.
constexpr int kScatterTile = 512;

__global__ void __launch_bounds__(kThreads) k_tadj_scatter(TParams P, BkState in, BkConstants cst, BkGridFields g,
                                                         BkAdjointTransport a, const BkAdjointState adj) {
    __shared__ double s_bar[4][kScatterTile];
    __shared__ int s_box[6];
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + tid;
    const int64_t pitch = P.pitch;
    Stencil st;
    st.valid = false;
    st.b[0] = st.b[1] = st.b[2] = 0;
    if (i < P.n) st = make_stencil(load_v3(in.x, i, pitch), P.origin, P.dx, P.R);
    const bool valid = i < P.n && st.valid;
    // the block's node box
    if (tid < 6) s_box[tid] = tid < 3 ? INT_MAX : INT_MIN;
    __syncthreads();
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int lo = __reduce_min_sync(0xffffffffu, valid ? st.b[ax] : INT_MAX);
        const int hi = __reduce_max_sync(0xffffffffu, valid ? st.b[ax] + 2 : INT_MIN);
        if (lane == 0 && lo != INT_MAX) {
            atomicMin(&s_box[ax], lo);
            atomicMax(&s_box[3 + ax], hi);
        }
    }
    __syncthreads();
    int lo[3] = {0, 0, 0}, ext[3] = {1, 1, 1};
    int count = 0;
    if (s_box[0] != INT_MAX) {
        long long c = 1;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            lo[ax] = s_box[ax];
            ext[ax] = s_box[3 + ax] - s_box[ax] + 1;
            c *= ext[ax];
        }
        count = c <= kScatterTile ? (int)c : 0;
    }
    for (int t = tid; t < count; t += kThreads) {
        const int z = t % ext[2], y = (t / ext[2]) % ext[1], x = t / (ext[2] * ext[1]);
        const int64_t node = node_index(lo[0] + x, lo[1] + y, lo[2] + z, P.R);
#pragma unroll
        for (int f = 0; f < 4; ++f) s_bar[f][t] = g.field_bar[f][node];
    }
    __syncthreads();  // uniform: every thread reaches it
    if (!valid) return;
    const M3 F = load_m3(in.F, i, pitch);
    const double vol = (double)cst.volume[i] * (double)det3(F);
    const double cap = cst.capacity[i], T = in.temperature[i], W = in.water[i];
    double volb = 0.0, Tb = 0.0, Wb = 0.0;
    const float inv_dx = 1.f / P.dx;
    float xg[3] = {0.f, 0.f, 0.f};
#pragma unroll 3
    for (int j = 0; j < 27; ++j) {
        int ox, oy, oz;
        node_offset(j, ox, oy, oz);
        float dw[3];
        const double w = (double)weight_and_grad(st, ox, oy, oz, inv_dx, dw);
        double f0, f1, f2, f3;
        if (count > 0) {
            const int t = ((st.b[0] + ox - lo[0]) * ext[1] + (st.b[1] + oy - lo[1])) * ext[2] + (st.b[2] + oz - lo[2]);
            f0 = s_bar[0][t]; f1 = s_bar[1][t]; f2 = s_bar[2][t]; f3 = s_bar[3][t];
        } else {
            const int64_t node = node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R);
            f0 = g.field_bar[0][node]; f1 = g.field_bar[1][node]; f2 = g.field_bar[2][node]; f3 = g.field_bar[3][node];
        }
        volb += w * f0;
        Tb += w * cap * f2;
        Wb += w * f3;
        const float sv = (float)(vol * f0 + cap * f1 + cap * T * f2 + W * f3);
#pragma unroll
        for (int c = 0; c < 3; ++c) xg[c] += dw[c] * sv;
    }
    a.temperature_in[i] += Tb;
    a.water_in[i] += Wb;
#pragma unroll
    for (int c = 0; c < 3; ++c) adj.x[c * pitch + i] += xg[c];
    add_det_grad(adj.F, i, pitch, F, (float)(volb * (double)cst.volume[i]));
}

// ---------------------------------------------------------------- surface
// Mesh vertex positions of this substep (geometry/mesh_tracking.py:13-38) into surface.vertices,
// as the forward's transport phase computes them (vertex_block: one block per boundary vertex).
template <int kBlock>
__global__ void __launch_bounds__(kBlock) k_tadj_vertex_positions(TParams P, const float* __restrict__ x,
                                                               const float* __restrict__ F, BkSurface sf) {
    const int vid = sf.vertex_ids[blockIdx.x];
    const float v = vertex_block<kBlock>(sf.binding_offsets, sf.binding_particles, sf.binding_weights,
                                           sf.reference_offsets, sf.binding_pitch, sf.reference_vertices,
                                           sf.vertex_pitch, x, F, P.pitch, vid);
    if (threadIdx.x < 3) sf.vertices[threadIdx.x * sf.vertex_pitch + vid] = v;
}

__device__ __forceinline__ void face_vertices(const BkSurface& sf, int f, double q[3][3], int vid[3]) {
    const int64_t vp = sf.vertex_pitch;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        vid[k] = sf.faces[3 * f + k];
#pragma unroll
        for (int a = 0; a < 3; ++a) q[k][a] = (double)sf.vertices[a * vp + vid[k]];
    }
}

__global__ void k_tadj_owners(TParams P, BkState in, BkConstants cst, BkSurface sf, BkGridFields g,
                              BkAdjointTransport a, const BkAdjointState adj) {
    const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (o >= sf.owner_count) return;
    const int64_t pitch = P.pitch;
    const int p = sf.owners[o];
    Stencil st = make_stencil(load_v3(in.x, p, pitch), P.origin, P.dx, P.R);
    if (!st.valid) return;
    // recompute the owner's exposed and tray-contact areas
    double exposed = 0.0, contact = 0.0;
    const int f0 = sf.owner_face_offsets[o], f1 = sf.owner_face_offsets[o + 1];
    for (int f = f0; f < f1; ++f) {
        double q[3][3];
        int vid[3];
        face_vertices(sf, f, q, vid);
        const double e1[3] = {q[1][0] - q[0][0], q[1][1] - q[0][1], q[1][2] - q[0][2]};
        const double e2[3] = {q[2][0] - q[0][0], q[2][1] - q[0][1], q[2][2] - q[0][2]};
        const double nr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double len = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
        const double cy = (q[0][1] + q[1][1] + q[2][1]) / 3.0;
        if (cy <= P.contact_limit && nr[1] < -0.2 * len) contact += 0.5 * len;
        else exposed += 0.5 * len;
    }
    const M3 F = load_m3(in.F, p, pitch);
    const double vol = (double)cst.volume[p] * (double)det3(F);
    const double T = in.temperature[p], W = in.water[p];
    const double sat = W / (P.rho_w * vol);
    const double h = (double)cst.heat_parameter[0];
    const double loss = P.water_enabled ? P.surface_loss * T * sat * exposed : 0.0;
    const double heat = h * exposed * (P.oven - T) + P.tray_transfer * contact * (P.tray - T) - P.latent * loss;
    // gather the heat and loss adjoints from the owner's stencil
    double heatb = 0.0, lossb = 0.0;
    const float inv_dx = 1.f / P.dx;
    float xg[3] = {0.f, 0.f, 0.f};
#pragma unroll 1
    for (int j = 0; j < 27; ++j) {
        int ox, oy, oz;
        node_offset(j, ox, oy, oz);
        float dw[3];
        const double w = (double)weight_and_grad(st, ox, oy, oz, inv_dx, dw);
        const int64_t node = node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R);
        const double fh = g.field_bar[4][node], fl = g.field_bar[5][node];
        heatb += w * fh;
        lossb += w * fl;
        const float s = (float)(heat * fh + loss * fl);
#pragma unroll
        for (int c = 0; c < 3; ++c) xg[c] += dw[c] * s;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) adj.x[c * pitch + p] += xg[c];
    const double lossb_all = lossb - P.latent * heatb;
    double Tb = heatb * (-h * exposed - P.tray_transfer * contact);
    double exposedb = heatb * h * (P.oven - T), contactb = heatb * P.tray_transfer * (P.tray - T);
    if (P.water_enabled) {
        Tb += lossb_all * P.surface_loss * sat * exposed;
        exposedb += lossb_all * P.surface_loss * T * sat;
        const double satb = lossb_all * P.surface_loss * T * exposed;
        a.water_in[p] += satb / (P.rho_w * vol);
        const double volb = -satb * sat / vol;
        add_det_grad(adj.F, p, pitch, F, (float)(volb * (double)cst.volume[p]));
    }
    a.temperature_in[p] += Tb;
    if (a.heat_parameter) atomicAdd(a.heat_parameter, heatb * exposed * (P.oven - T));
    // face areas -> vertex adjoints
    const int64_t vp = sf.vertex_pitch;
    for (int f = f0; f < f1; ++f) {
        double q[3][3];
        int vid[3];
        face_vertices(sf, f, q, vid);
        const double e1[3] = {q[1][0] - q[0][0], q[1][1] - q[0][1], q[1][2] - q[0][2]};
        const double e2[3] = {q[2][0] - q[0][0], q[2][1] - q[0][1], q[2][2] - q[0][2]};
        const double nr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const double len = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
        if (!(len > 0.0)) continue;
        const double cy = (q[0][1] + q[1][1] + q[2][1]) / 3.0;
        const bool is_contact = cy <= P.contact_limit && nr[1] < -0.2 * len;
        const double areab = is_contact ? contactb : exposedb;
        // area = |e1 x e2| / 2: nbar = areab n / (2 |n|); e1bar = e2 x nbar, e2bar = nbar x e1
        const double k = areab * 0.5 / len;
        const double nb[3] = {k * nr[0], k * nr[1], k * nr[2]};
        const double e1b[3] = {e2[1] * nb[2] - e2[2] * nb[1], e2[2] * nb[0] - e2[0] * nb[2], e2[0] * nb[1] - e2[1] * nb[0]};
        const double e2b[3] = {nb[1] * e1[2] - nb[2] * e1[1], nb[2] * e1[0] - nb[0] * e1[2], nb[0] * e1[1] - nb[1] * e1[0]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            atomicAdd(&a.vertices[c * vp + vid[0]], -(e1b[c] + e2b[c]));
            atomicAdd(&a.vertices[c * vp + vid[1]], e1b[c]);
            atomicAdd(&a.vertices[c * vp + vid[2]], e2b[c]);
        }
    }
}

// One block per surface vertex: its adjoint to the bound particles' x and F, then zeroed.
template <int kBlock>
__global__ void __launch_bounds__(kBlock) k_tadj_vertices(TParams P, BkSurface sf, BkAdjointTransport a,
                                                       const BkAdjointState adj) {
    __shared__ float s_w[kBlock / 32];
    const int vid = sf.vertex_ids[blockIdx.x];
    const int t = threadIdx.x;
    const int64_t vp = sf.vertex_pitch, bp = sf.binding_pitch, pitch = P.pitch;
    const double vb[3] = {a.vertices[vid], a.vertices[vp + vid], a.vertices[2 * vp + vid]};
    __syncthreads();
    if (t < 3) a.vertices[t * vp + vid] = 0.0;
    const int b0 = sf.binding_offsets[vid], b1 = sf.binding_offsets[vid + 1];
    if (b0 == b1 || (vb[0] == 0.0 && vb[1] == 0.0 && vb[2] == 0.0)) return;  // the same for the whole block
    // v = (1 - sum_b w_b) pred_b0 + sum_b w_b pred_b
    float wsum = 0.f;
    for (int b = b0 + t; b < b1; b += kBlock) wsum += sf.binding_weights[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((t & 31) == 0) s_w[t >> 5] = wsum;
    __syncthreads();
    wsum = 0.f;
    for (int w = 0; w < kBlock / 32; ++w) wsum += s_w[w];
    for (int b = b0 + t; b < b1; b += kBlock) {
        const float c = sf.binding_weights[b] + (b == b0 ? 1.f - wsum : 0.f);
        const int p = sf.binding_particles[b];
        const float o[3] = {sf.reference_offsets[b], sf.reference_offsets[bp + b], sf.reference_offsets[2 * bp + b]};
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const float pb = (float)(c * vb[r]);
            atomicAdd(&adj.x[r * pitch + p], pb);
#pragma unroll
            for (int k = 0; k < 3; ++k) atomicAdd(&adj.F[(3 * r + k) * pitch + p], pb * o[k]);
        }
    }
}

// ------------------------------------------------------------------- clear
__global__ void k_tadj_clear(TParams P, BkGridFields g, const int32_t* __restrict__ box) {
    int lo[3], ext[3];
    int64_t count = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int l = max(box[k], 0), h = min(box[3 + k], P.R - 1);
        if (l > h) return;
        lo[k] = l;
        ext[k] = h - l + 1;
        count *= ext[k];
    }
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
        const int c2 = lo[2] + (int)(t % ext[2]);
        const int c1 = lo[1] + (int)((t / ext[2]) % ext[1]);
        const int c0 = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        const int64_t i = node_index(c0, c1, c2, P.R);
#pragma unroll
        for (int k = 0; k < 7; ++k) g.fields[k][i] = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) g.field_bar[k][i] = 0.0;
        g.dTr_bar[i] = make_double2(0.0, 0.0);
    }
}

TParams tparams(const BkSubstepParams& p, const BkSurface* sf) {
    TParams t;
    t.n = p.n; t.pitch = p.pitch; t.R = p.resolution;
    for (int k = 0; k < 3; ++k) t.origin[k] = p.origin[k];
    t.dx = p.spacing; t.dt = p.time_step;
    t.rho_w = p.scalar.water_density;
    t.s0 = p.initial_saturation;
    t.c_water = p.water_stress;
    t.kc = (double)(p.conductivity * p.spacing);
    t.kw = (double)(p.diffusivity * p.scalar.water_density * p.spacing);
    t.cell = (double)(p.spacing * p.spacing * p.spacing);
    t.water_enabled = p.scalar.water_enabled;
    t.oven = p.scalar.oven_temperature; t.tray = p.scalar.tray_temperature;
    t.tray_transfer = p.scalar.tray_transfer; t.surface_loss = p.scalar.surface_loss; t.latent = p.scalar.latent_heat;
    t.contact_limit = sf ? (double)(sf->floor_height + sf->contact_distance) : 0.0;
    t.gas = p.gas;
    t.settling = p.settling;
    t.ambient = p.gas_ambient_pressure;
    t.peak = p.gas_peak;
    t.width = p.gas_width;
    t.source_scale = (double)(p.time_step * p.density);
    return t;
}

unsigned blocks(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

extern "C" {

int bk_transport_adjoint_prepare(const BkSubstepParams* params, const BkState* in, const BkConstants* constants,
                                 const double* node_dT_ratio, float* material_temperature, float* mass,
                                 float* stress, void* stream) {
    if (!params || !in || !constants || !node_dT_ratio || !material_temperature || !mass || !stress)
        return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint_prepare: null argument");
    const BkSubstepParams& p = *params;
    if (!p.transport || p.material != 1 || !in->temperature || !in->water || !in->tau || !constants->dry_mass)
        return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint_prepare: needs the Ding model with transport");
    if (p.gas && (!in->gas_moles || !in->porosity || !constants->gas_rate))
        return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint_prepare: gas mode needs the gas arrays");
    if (p.n == 0) return BK_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_tadj_prepare<<<blocks(p.n, 256), 256, 0, s>>>(tparams(p, nullptr), *in, *constants,
                                                    reinterpret_cast<const double2*>(node_dT_ratio),
                                                    material_temperature, mass, stress);
    return check_launch("bk_transport_adjoint_prepare");
}

int bk_transport_adjoint(const BkSubstepParams* params, const BkState* in, const BkConstants* constants,
                         const BkGrid* grid, const BkSurface* surface, const BkAdjointState* mechanics,
                         BkAdjointTransport* adjoint, void* stream) {
    if (!params || !in || !constants || !grid || !surface || !mechanics || !adjoint)
        return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint: null argument");
    const BkSubstepParams& p = *params;
    if (!p.transport || p.material != 1)
        return fail(BK_ERR_UNSUPPORTED, "bk_transport_adjoint: the Ding model with transport");
    if (p.gas && (!in->gas_moles || !in->porosity || !constants->gas_rate || !adjoint->gas_moles_out ||
                  !adjoint->gas_moles_in || !mechanics->porosity))
        return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint: gas mode needs the gas arrays and their adjoints");
    const BkAdjointTransport& a = *adjoint;
    if (!a.temperature_out || !a.water_out || !a.temperature_in || !a.water_in || !a.node_dT_ratio || !a.vertices ||
        !mechanics->tau || !mechanics->mass || !mechanics->temperature || !mechanics->x || !mechanics->F)
        return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint: missing adjoint arrays");
    for (int k = 0; k < 6; ++k)
        if (!a.node_fields[k]) return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint: missing node-field adjoint");
    for (int k = 0; k < 7; ++k)
        if (!grid->fields[k]) return fail(BK_ERR_ARGUMENT, "bk_transport_adjoint: missing node field");
    if (p.n == 0) return BK_OK;
    const TParams P = tparams(p, surface);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    BkGridFields g;
    for (int k = 0; k < 7; ++k) g.fields[k] = grid->fields[k];
    for (int k = 0; k < 6; ++k) g.field_bar[k] = a.node_fields[k];
    g.dTr_bar = reinterpret_cast<double2*>(a.node_dT_ratio);
    const int32_t* box = grid->bounds + 6;
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const unsigned box_blocks = (unsigned)sms * 4;
    k_tadj_scalar<<<blocks(p.n, kThreads), kThreads, 0, s>>>(P, *in, *constants,
                                                             reinterpret_cast<const double2*>(grid->node_dT_ratio), a,
                                                             *mechanics, g.dTr_bar);
    if (int rc = check_launch("bk_transport_adjoint/scalar")) return rc;
    k_tadj_diffuse<<<box_blocks, 256, 0, s>>>(P, g, box);
    if (int rc = check_launch("bk_transport_adjoint/diffuse")) return rc;
    k_tadj_scatter<<<blocks(p.n, kThreads), kThreads, 0, s>>>(P, *in, *constants, g, a, *mechanics);
    if (int rc = check_launch("bk_transport_adjoint/scatter")) return rc;
    if (surface->vertex_count > 0) {
        const unsigned nv = (unsigned)surface->vertex_count;
        switch (vertex_block_threads(surface->vertex_count, surface->binding_count)) {
            case 256: k_tadj_vertex_positions<256><<<nv, 256, 0, s>>>(P, in->x, in->F, *surface); break;
            case 128: k_tadj_vertex_positions<128><<<nv, 128, 0, s>>>(P, in->x, in->F, *surface); break;
            default: k_tadj_vertex_positions<32><<<nv, 32, 0, s>>>(P, in->x, in->F, *surface); break;
        }
        if (int rc = check_launch("bk_transport_adjoint/vertex_positions")) return rc;
    }
    if (surface->owner_count > 0) {
        k_tadj_owners<<<blocks(surface->owner_count, 64), 64, 0, s>>>(P, *in, *constants, *surface, g, a, *mechanics);
        if (int rc = check_launch("bk_transport_adjoint/owners")) return rc;
    }
    if (surface->vertex_count > 0) {
        const unsigned nv = (unsigned)surface->vertex_count;
        switch (vertex_block_threads(surface->vertex_count, surface->binding_count)) {
            case 256: k_tadj_vertices<256><<<nv, 256, 0, s>>>(P, *surface, a, *mechanics); break;
            case 128: k_tadj_vertices<128><<<nv, 128, 0, s>>>(P, *surface, a, *mechanics); break;
            default: k_tadj_vertices<32><<<nv, 32, 0, s>>>(P, *surface, a, *mechanics); break;
        }
        if (int rc = check_launch("bk_transport_adjoint/vertices")) return rc;
    }
    k_tadj_clear<<<box_blocks, 256, 0, s>>>(P, g, box);
    return check_launch("bk_transport_adjoint/clear");
}

}  // extern "C"
