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

__global__ void k_measure_finish(const double* __restrict__ partial, double* __restrict__ out, int blocks,
                                 int has_ding, int has_gas, int has_transport, int has_mesh) {
    const int s = threadIdx.x;
    if (s >= kSlots) return;
    const int op = slot_op(s);
    double v = partial[s];
    for (int b = 1; b < blocks; ++b) v = combine(op, v, partial[(int64_t)b * kSlots + s]);
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
    const int k = threadIdx.x;
    if (k >= 2) return;
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += partial[2 * b + k];
    out[k] = v;
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
    k_step_summary_finish<<<1, 32, 0, s>>>(scratch, out, BK_MEASURE_BLOCKS);
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
    k_measure_finish<<<1, 64, 0, s>>>(scratch, out, BK_MEASURE_BLOCKS, m.porosity != nullptr, m.gas_moles != nullptr,
                                      m.temperature != nullptr, m.vertex_count > 0);
    return check_launch("bk_measure_state/finish");
}
