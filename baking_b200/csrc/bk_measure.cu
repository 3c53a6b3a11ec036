// The recorder's per-step measurements (experiments/recording.py:46-112) as one device reduction:
// every block strides over the particles, the mesh vertices and the tets, keeps per-thread sums,
// minima and maxima in registers, reduces them across the block and writes one partial per slot;
// a one-block pass then reduces the BK_MEASURE_BLOCKS partials of each slot in a fixed order, so
// the result does not depend on scheduling. The host reads BK_MEASURE_SLOTS doubles instead of
// every state array.
#include <cmath>
#include <cstdint>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"

using namespace bk;

namespace {

constexpr int kThreads = 256;
constexpr int kSlots = BK_MEASURE_SLOTS;

enum Op { kSum = 0, kMin = 1, kMax = 2 };

__host__ __device__ constexpr int slot_op(int s) {
    return (s == BK_MEASURE_POROSITY_MIN || s == BK_MEASURE_PRESSURE_MIN || s == BK_MEASURE_T_MIN ||
            s == BK_MEASURE_SATURATION_MIN || s == BK_MEASURE_X_MIN || s == BK_MEASURE_Y_MIN || s == BK_MEASURE_Z_MIN)
               ? kMin
               : (s == BK_MEASURE_POROSITY_MAX || s == BK_MEASURE_PRESSURE_MAX || s == BK_MEASURE_T_MAX ||
                  s == BK_MEASURE_SATURATION_MAX || s == BK_MEASURE_X_MAX || s == BK_MEASURE_Y_MAX ||
                  s == BK_MEASURE_Z_MAX)
                     ? kMax
                     : kSum;
}

__device__ __forceinline__ double slot_init(int s) {
    const int op = slot_op(s);
    return op == kMin ? INFINITY : (op == kMax ? -INFINITY : 0.0);
}

__device__ __forceinline__ double combine(int op, double a, double b) {
    return op == kMin ? fmin(a, b) : (op == kMax ? fmax(a, b) : a + b);
}

__device__ __forceinline__ void add(double* acc, int s, double v) {
    acc[s] = combine(slot_op(s), acc[s], v);
}

__global__ void __launch_bounds__(kThreads) k_measure(BkMeasureInputs in, double* __restrict__ partial) {
    double acc[kSlots];
#pragma unroll
    for (int s = 0; s < kSlots; ++s) acc[s] = slot_init(s);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t pitch = in.pitch;
    for (int64_t i = first; i < in.n; i += stride) {
        double F[9];
        bool finite = true;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const float f = in.F[e * pitch + i];
            finite = finite && isfinite(f);
            F[e] = (double)f;
        }
        if (!finite) add(acc, BK_MEASURE_NONFINITE, 1.0);
        const double J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                         F[2] * (F[3] * F[7] - F[4] * F[6]);
        const double V0 = (double)in.reference_volume[i];
        add(acc, BK_MEASURE_PARTICLE_VOLUME, V0 * J);
        if (J <= 0.0) add(acc, BK_MEASURE_INVALID_PARTICLES, 1.0);
        if (in.porosity) {
            const double n = (double)in.porosity[i];
            add(acc, BK_MEASURE_MATERIAL_T_SUM, (double)in.material_temperature[i]);
            add(acc, BK_MEASURE_POROSITY_SUM, n);
            add(acc, BK_MEASURE_POROSITY_MIN, n);
            add(acc, BK_MEASURE_POROSITY_MAX, n);
            if (in.gelled[i]) add(acc, BK_MEASURE_GELLED, 1.0);
            if (in.gas_moles) {
                const double p = in.gas_pressure[i];
                add(acc, BK_MEASURE_GAS_TOTAL, V0 * in.gas_moles[i]);
                add(acc, BK_MEASURE_PRESSURE_SUM, p);
                add(acc, BK_MEASURE_PRESSURE_MIN, p);
                add(acc, BK_MEASURE_PRESSURE_MAX, p);
                add(acc, BK_MEASURE_PORE_VOLUME, V0 * J * n);
            }
        }
        if (in.temperature) {
            const double T = in.temperature[i], c = in.capacity[i], s = in.saturation[i];
            add(acc, BK_MEASURE_T_MIN, T);
            add(acc, BK_MEASURE_T_MAX, T);
            add(acc, BK_MEASURE_ENERGY, c * T);
            add(acc, BK_MEASURE_CAPACITY, c);
            const uint8_t r = in.regions[i];
            if (r & 1) {
                add(acc, BK_MEASURE_SURFACE_T_SUM, T);
                add(acc, BK_MEASURE_SURFACE_COUNT, 1.0);
            }
            if (r & 2) {
                add(acc, BK_MEASURE_CORE_T_SUM, T);
                add(acc, BK_MEASURE_CORE_COUNT, 1.0);
            }
            add(acc, BK_MEASURE_WATER, in.water[i]);
            add(acc, BK_MEASURE_WATER_LOST, in.water_losses[i]);
            add(acc, BK_MEASURE_HEAT_EXCHANGE, in.heat_exchanges[i]);
            add(acc, BK_MEASURE_SATURATION_SUM, s);
            add(acc, BK_MEASURE_SATURATION_MIN, s);
            add(acc, BK_MEASURE_SATURATION_MAX, s);
        }
    }
    const int64_t vp = in.vertex_pitch;
    for (int64_t v = first; v < in.vertex_count; v += stride) {
        const float x = in.vertices[v], y = in.vertices[vp + v], z = in.vertices[2 * vp + v];
        if (!(isfinite(x) && isfinite(y) && isfinite(z))) add(acc, BK_MEASURE_NONFINITE, 1.0);
        add(acc, BK_MEASURE_X_MIN, (double)x);
        add(acc, BK_MEASURE_Y_MIN, (double)y);
        add(acc, BK_MEASURE_Z_MIN, (double)z);
        add(acc, BK_MEASURE_X_MAX, (double)x);
        add(acc, BK_MEASURE_Y_MAX, (double)y);
        add(acc, BK_MEASURE_Z_MAX, (double)z);
    }
    for (int64_t t = first; t < in.tet_count; t += stride) {
        double c[4][3];
        bool inside = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int64_t v = in.tets[4 * t + k];
            if (v < 0 || v >= in.vertex_count) {
                inside = false;  // a corrupt tet: counted, not read
                v = 0;
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) c[k][a] = (double)in.vertices[a * vp + v];
        }
        if (!inside) {
            add(acc, BK_MEASURE_NONFINITE, 1.0);
            continue;
        }
        double e[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int a = 0; a < 3; ++a) e[k][a] = c[k + 1][a] - c[0][a];
        // det of the edge rows / 6 (geometry/mesh_validation.py ComputeSignedVolumes)
        const double vol = (e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                            e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                            e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0])) / 6.0;
        add(acc, BK_MEASURE_MESH_VOLUME, fabs(vol));
        if (vol <= 0.0) add(acc, BK_MEASURE_INVERTED_TETS, 1.0);
    }
    // block reduction, one slot at a time
    __shared__ double s_warp[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < kSlots; ++s) {
        const int op = slot_op(s);
        double v = acc[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = combine(op, v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) s_warp[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = s_warp[0];
            for (int w = 1; w < kThreads / 32; ++w) b = combine(op, b, s_warp[w]);
            partial[(int64_t)blockIdx.x * kSlots + s] = b;
        }
        __syncthreads();
    }
}

// One slot's block partials reduced by one warp: lane l combines partials l, l + 32, ... in that
// order, then a fixed butterfly combines the lanes (a deterministic order, whatever the schedule).
__device__ __forceinline__ double warp_slot_reduce(int op, const double* __restrict__ partial, int blocks, int stride,
                                                   int slot) {
    const int lane = threadIdx.x & 31;
    double v = op == kMin ? INFINITY : (op == kMax ? -INFINITY : 0.0);
    for (int b = lane; b < blocks; b += 32) v = combine(op, v, partial[(int64_t)b * stride + slot]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = combine(op, v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__global__ void k_measure_finish(const double* __restrict__ partial, double* __restrict__ out, int blocks,
                                 int has_ding, int has_gas, int has_transport, int has_mesh) {
    const int s = blockIdx.x;  // one warp per slot
    const int op = slot_op(s);
    double v = warp_slot_reduce(op, partial, blocks, kSlots, s);
    if (threadIdx.x != 0) return;
    const bool ding = s >= BK_MEASURE_MATERIAL_T_SUM && s <= BK_MEASURE_GELLED;
    const bool gas = s >= BK_MEASURE_GAS_TOTAL && s <= BK_MEASURE_PORE_VOLUME;
    const bool transport = s >= BK_MEASURE_T_MIN && s <= BK_MEASURE_SATURATION_MAX;
    const bool mesh = s >= BK_MEASURE_X_MIN && s <= BK_MEASURE_Z_MAX;
    if ((ding && !has_ding) || (gas && !has_gas) || (transport && !has_transport) || (mesh && !has_mesh)) v = 0.0;
    out[s] = v;
}

// Step result: the grid mass of the last substep (node masses over its active box, the only
// nonzero nodes) and the particles' kinetic energy sum 1/2 m |v|^2 with m = dry + W under
// transport, in two deterministic passes like k_measure.
__global__ void __launch_bounds__(kThreads) k_step_summary(int64_t n, int64_t pitch, const float* __restrict__ v,
                                                         const float* __restrict__ mass, const double* __restrict__ dry,
                                                         const double* __restrict__ water, const float4* __restrict__ pm,
                                                         const int32_t* __restrict__ box, int R,
                                                         double* __restrict__ partial) {
    double grid = 0.0, kinetic = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t i = first; i < n; i += stride) {
        const double m = water ? dry[i] + water[i] : (double)mass[i];
        const double a = v[i], b = v[pitch + i], c = v[2 * pitch + i];
        kinetic += 0.5 * m * (a * a + b * b + c * c);
    }
    int lo[3], ext[3];
    int64_t count = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int l = max(box[k], 0), h = min(box[3 + k], R - 1);
        lo[k] = l;
        ext[k] = h >= l ? h - l + 1 : 0;
        count *= ext[k];
    }
    for (int64_t t = first; t < count; t += stride) {
        const int z = lo[2] + (int)(t % ext[2]);
        const int y = lo[1] + (int)((t / ext[2]) % ext[1]);
        const int x = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        grid += (double)pm[node_index(x, y, z, R)].w;
    }
    __shared__ double s_warp[2][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        grid += __shfl_xor_sync(0xffffffffu, grid, o);
        kinetic += __shfl_xor_sync(0xffffffffu, kinetic, o);
    }
    if (lane == 0) {
        s_warp[0][warp] = grid;
        s_warp[1][warp] = kinetic;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double b = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) b += s_warp[threadIdx.x][w];
        partial[2 * (int64_t)blockIdx.x + threadIdx.x] = b;
    }
}

__global__ void k_step_summary_finish(const double* __restrict__ partial, double* __restrict__ out, int blocks) {
    const int k = blockIdx.x;  // one warp per value
    const double v = warp_slot_reduce(kSum, partial, blocks, 2, k);
    if (threadIdx.x == 0) out[k] = v;
}

// ------------------------------------------------------------------ CheckState
// physics/mpm.py:243-308 as one reduction; slots and their meaning are BK_CHECK_* of the header.
constexpr int kCheckSlots = BK_CHECK_SLOTS;

__host__ __device__ constexpr int check_op(int s) {
    return s == BK_CHECK_J_MIN ? kMin
           : (s == BK_CHECK_J_MAX || s == BK_CHECK_SPEED_MAX || s == BK_CHECK_GAS_WAVE_MAX ||
              s == BK_CHECK_WATER_WAVE2_MAX || s == BK_CHECK_RESIDUAL_MAX || s <= BK_CHECK_TRANSPORT_FLAG1)
                 ? kMax
                 : kSum;
}

__device__ __forceinline__ void check_add(double* acc, int s, double v) { acc[s] = combine(check_op(s), acc[s], v); }

__global__ void __launch_bounds__(kThreads) k_check_state(BkCheckInputs in, double* __restrict__ partial) {
    double acc[kCheckSlots];
#pragma unroll
    for (int s = 0; s < kCheckSlots; ++s) {
        const int op = check_op(s);
        acc[s] = op == kMin ? INFINITY : (op == kMax ? -INFINITY : 0.0);
    }
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t pitch = in.pitch;
    const double inv_dx = 1.0 / (double)in.spacing;
    const double hi = (double)in.resolution - 1.5;
    for (int64_t i = first; i < in.n; i += stride) {
        bool finite = true;
        double x[3], v[3], F[9];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float xa = in.x[a * pitch + i], va = in.v[a * pitch + i];
            finite = finite && isfinite(xa) && isfinite(va);
            x[a] = xa;
            v[a] = va;
        }
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const float f = in.F[e * pitch + i], c = in.C[e * pitch + i];
            finite = finite && isfinite(f) && isfinite(c);
            F[e] = f;
        }
        if (!finite) check_add(acc, BK_CHECK_NONFINITE_STATE, 1.0);
        const double J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                         F[2] * (F[3] * F[7] - F[4] * F[6]);
        check_add(acc, BK_CHECK_J_MIN, J);
        check_add(acc, BK_CHECK_J_MAX, J);
        bool outside = false;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double g = (x[a] - (double)in.origin[a]) * inv_dx;
            outside = outside || g < 0.5 || g >= hi;
        }
        if (outside) check_add(acc, BK_CHECK_OUTSIDE_STENCIL, 1.0);
        const double speed2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        check_add(acc, BK_CHECK_SPEED_MAX, sqrt(speed2));
        const double V0 = (double)in.reference_volume[i];
        check_add(acc, BK_CHECK_PARTICLE_VOLUME, V0 * J);
        const double m = in.water ? in.dry_mass[i] + in.water[i] : (double)in.mass[i];
        check_add(acc, BK_CHECK_TOTAL_MASS, m);
        check_add(acc, BK_CHECK_KINETIC_ENERGY, 0.5 * m * speed2);
        const double rho = in.water ? m / V0 : (double)in.density;
        if (in.gas_moles) {
            const double n = (double)in.porosity[i];
            const float T = in.temperature ? (float)in.temperature[i] : in.material_temperature[i];
            const double p = gas_pressure(in.gas_moles[i], T, (float)J, (float)n);
            const double bulk = p * (1.0 + (1.0 - (double)in.initial_porosity + n) / n);
            check_add(acc, BK_CHECK_GAS_WAVE_MAX, sqrt(((double)in.gas_modulus + bulk) * J / rho));
        }
        if (in.water && in.water_enabled) {
            const double sat = in.water[i] / ((double)in.water_density * V0 * J);
            check_add(acc, BK_CHECK_WATER_WAVE2_MAX, (double)in.water_stress * sat * J / rho);
        }
        if (in.Fe) {
            M3 Fe, Ff;
            bool ok = true;
#pragma unroll
            for (int e = 0; e < 9; ++e) {
                Fe.m[e] = in.Fe[e * pitch + i];
                Ff.m[e] = (float)F[e];
                ok = ok && isfinite(Fe.m[e]);
            }
            if (ok) {
                const M3 Fp = matmul(inverse3(Fe), Ff);
#pragma unroll
                for (int e = 0; e < 9; ++e) ok = ok && isfinite(Fp.m[e]);
            }
            if (!ok) check_add(acc, BK_CHECK_NONFINITE_DING, 1.0);
            if (in.return_residuals) check_add(acc, BK_CHECK_RESIDUAL_MAX, (double)in.return_residuals[i]);
        }
    }
    if (in.node_pm && in.box) {
        int lo[3], ext[3];
        int64_t count = 1;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int l = max(in.box[k], 0), h = min(in.box[3 + k], in.resolution - 1);
            lo[k] = l;
            ext[k] = h >= l ? h - l + 1 : 0;
            count *= ext[k];
        }
        const float4* pm = reinterpret_cast<const float4*>(in.node_pm);
        for (int64_t t = first; t < count; t += stride) {
            const int z = lo[2] + (int)(t % ext[2]);
            const int y = lo[1] + (int)((t / ext[2]) % ext[1]);
            const int xx = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
            check_add(acc, BK_CHECK_GRID_MASS, (double)pm[node_index(xx, y, z, in.resolution)].w);
        }
    }
    const int64_t vp = in.vertex_pitch;
    for (int64_t q = first; q < in.vertex_count; q += stride) {
        const float a = in.vertices[q], b = in.vertices[vp + q], c = in.vertices[2 * vp + q];
        if (!(isfinite(a) && isfinite(b) && isfinite(c))) check_add(acc, BK_CHECK_NONFINITE_VERTICES, 1.0);
    }
    for (int64_t t = first; t < in.tet_count; t += stride) {
        double c[4][3];
        bool inside = true;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int64_t q = in.tets[4 * t + k];
            if (q < 0 || q >= in.vertex_count) {
                inside = false;
                q = 0;
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) c[k][a] = (double)in.vertices[a * vp + q];
        }
        double e[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int a = 0; a < 3; ++a) e[k][a] = c[k + 1][a] - c[0][a];
        const double vol = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                           e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                           e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
        if (!inside || vol <= 0.0) check_add(acc, BK_CHECK_INVERTED_TETS, 1.0);
    }
    __shared__ double s_warp[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s < kCheckSlots; ++s) {
        const int op = check_op(s);
        double v = acc[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = combine(op, v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) s_warp[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = s_warp[0];
            for (int w = 1; w < kThreads / 32; ++w) b = combine(op, b, s_warp[w]);
            partial[(int64_t)blockIdx.x * kCheckSlots + s] = b;
        }
        __syncthreads();
    }
}

__global__ void k_check_finish(const double* __restrict__ partial, double* __restrict__ out, int blocks,
                               BkCheckInputs in) {
    const int s = blockIdx.x;  // one warp per slot
    const int op = check_op(s);
    double v = warp_slot_reduce(op, partial, blocks, kCheckSlots, s);
    if (threadIdx.x != 0) return;
    if (s == BK_CHECK_SIM_FLAG0 || s == BK_CHECK_SIM_FLAG1) v = (double)in.sim_flags[s - BK_CHECK_SIM_FLAG0];
    if (s >= BK_CHECK_DING_FLAG0 && s <= BK_CHECK_DING_FLAG2)
        v = in.ding_flags ? (double)in.ding_flags[s - BK_CHECK_DING_FLAG0] : 0.0;
    if (s == BK_CHECK_SUBSTEP_STATUS) v = in.substep_status ? (double)in.substep_status[0] : 0.0;
    if (s == BK_CHECK_TRANSPORT_FLAG0 || s == BK_CHECK_TRANSPORT_FLAG1)
        v = in.transport_flags ? (double)in.transport_flags[s - BK_CHECK_TRANSPORT_FLAG0] : 0.0;
    if (s == BK_CHECK_RESIDUAL_MAX) {
        if (in.max_residuals) v = fmax(v, (double)in.max_residuals[0]);
        if (!in.Fe) v = 0.0;
        v = fmax(v, 0.0);
    }
    if ((s == BK_CHECK_GAS_WAVE_MAX && !in.gas_moles) || (s == BK_CHECK_WATER_WAVE2_MAX && !(in.water && in.water_enabled)))
        v = 0.0;
    if (in.n == 0 && (s == BK_CHECK_J_MIN || s == BK_CHECK_J_MAX || s == BK_CHECK_SPEED_MAX)) v = 0.0;
    out[s] = v;
}

}  // namespace

extern "C" int bk_step_summary(const BkSubstepParams* params, const BkState* state, const BkConstants* constants,
                               const BkGrid* grid, double* out, double* scratch, void* stream) {
    if (!params || !state || !constants || !grid || !out || !scratch)
        return fail(BK_ERR_ARGUMENT, "bk_step_summary: null argument");
    const BkSubstepParams& p = *params;
    if (!state->v || !grid->node_pm || !grid->bounds || (p.transport ? (!constants->dry_mass || !state->water)
                                                                      : !constants->mass))
        return fail(BK_ERR_ARGUMENT, "bk_step_summary: missing arrays");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_step_summary<<<BK_MEASURE_BLOCKS, kThreads, 0, s>>>(p.n, p.pitch, state->v, constants->mass, constants->dry_mass,
                                                          p.transport ? state->water : nullptr,
                                                          reinterpret_cast<const float4*>(grid->node_pm),
                                                          grid->bounds + 6, p.resolution, scratch);
    if (int rc = check_launch("bk_step_summary")) return rc;
    k_step_summary_finish<<<2, 32, 0, s>>>(scratch, out, BK_MEASURE_BLOCKS);
    return check_launch("bk_step_summary/finish");
}

extern "C" int bk_measure_state(const BkMeasureInputs* in, double* out, double* scratch, void* stream) {
    if (!in || !out || !scratch) return fail(BK_ERR_ARGUMENT, "bk_measure_state: null argument");
    const BkMeasureInputs& m = *in;
    if (m.n < 0 || m.vertex_count < 0 || m.tet_count < 0 || (m.n > 0 && (m.pitch < m.n || !m.F || !m.reference_volume)))
        return fail(BK_ERR_ARGUMENT, "bk_measure_state: bad particle arrays");
    if (m.porosity && (!m.material_temperature || !m.gelled))
        return fail(BK_ERR_ARGUMENT, "bk_measure_state: Ding arrays incomplete");
    if (m.gas_moles && (!m.gas_pressure || !m.porosity))
        return fail(BK_ERR_ARGUMENT, "bk_measure_state: gas arrays incomplete");
    if (m.temperature && (!m.water || !m.saturation || !m.water_losses || !m.heat_exchanges || !m.capacity || !m.regions))
        return fail(BK_ERR_ARGUMENT, "bk_measure_state: transport arrays incomplete");
    if (m.vertex_count > 0 && (!m.vertices || m.vertex_pitch < m.vertex_count))
        return fail(BK_ERR_ARGUMENT, "bk_measure_state: bad vertex array");
    if (m.tet_count > 0 && (!m.tets || m.vertex_count == 0)) return fail(BK_ERR_ARGUMENT, "bk_measure_state: bad tets");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_measure<<<BK_MEASURE_BLOCKS, kThreads, 0, s>>>(m, scratch);
    if (int rc = check_launch("bk_measure_state")) return rc;
    k_measure_finish<<<kSlots, 32, 0, s>>>(scratch, out, BK_MEASURE_BLOCKS, m.porosity != nullptr, m.gas_moles != nullptr,
                                      m.temperature != nullptr, m.vertex_count > 0);
    return check_launch("bk_measure_state/finish");
}

extern "C" int bk_check_state(const BkCheckInputs* in, double* out, double* scratch, void* stream) {
    if (!in || !out || !scratch) return fail(BK_ERR_ARGUMENT, "bk_check_state: null argument");
    const BkCheckInputs& c = *in;
    if (c.n < 0 || c.vertex_count < 0 || c.tet_count < 0 || !c.sim_flags)
        return fail(BK_ERR_ARGUMENT, "bk_check_state: bad counts or missing flags");
    if (c.n > 0 && (c.pitch < c.n || !c.x || !c.v || !c.F || !c.C || !c.reference_volume ||
                    (c.water ? !c.dry_mass : !c.mass)))
        return fail(BK_ERR_ARGUMENT, "bk_check_state: bad particle arrays");
    if (c.gas_moles && (!c.porosity || !(c.temperature || c.material_temperature)))
        return fail(BK_ERR_ARGUMENT, "bk_check_state: gas arrays incomplete");
    if (!(c.spacing > 0.0f) || c.resolution < 1) return fail(BK_ERR_ARGUMENT, "bk_check_state: bad grid");
    if (c.node_pm && (!c.box || ((uintptr_t)c.node_pm & 15) != 0))
        return fail(BK_ERR_ARGUMENT, "bk_check_state: grid needs its active box and 16-byte alignment");
    if (c.vertex_count > 0 && (!c.vertices || c.vertex_pitch < c.vertex_count))
        return fail(BK_ERR_ARGUMENT, "bk_check_state: bad vertex array");
    if (c.tet_count > 0 && (!c.tets || c.vertex_count == 0)) return fail(BK_ERR_ARGUMENT, "bk_check_state: bad tets");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_check_state<<<BK_MEASURE_BLOCKS, kThreads, 0, s>>>(c, scratch);
    if (int rc = check_launch("bk_check_state")) return rc;
    k_check_finish<<<kCheckSlots, 32, 0, s>>>(scratch, out, BK_MEASURE_BLOCKS, c);
    return check_launch("bk_check_state/finish");
}
