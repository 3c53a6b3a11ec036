// Fused MLS-MPM baking substep for sm_100a (the simulator's hot path).
//
// The reference runs ~16 Warp launches per substep (physics/mpm.py:163-225,
// physics/thermal_water.py:296-367) with three host synchronisations and fresh
// dense-grid allocations. Here one substep is eight launches, clear_previous (which zeroes the last
// substep's momentum box) and these seven:
//
//   surface_vertices   rebuild only the boundary-face vertices (a block of 32-256 threads per
//                      vertex, sized by its mean particle bindings)
//   surface_owners     face areas -> boundary heat/loss/exchange of face-owning particles, scattered
//   transport_scatter  scalar P2G (volume, capacity, energy, water), warp-cooperative per stencil base
//   diffuse            7-point finite-volume heat/water flux over the active node box only
//   p2g                scalar G2P + gas source + gas/water stress + momentum P2G, fused per particle
//   grid_update        momentum -> velocity with walls over the active box; zeroes the scatter fields
//   g2p_return         G2P (v, C, x, F) fused with the Ding return map (float64 SVD in registers)
//
// Scatter scheme ("warp-cooperative stencil runs"): a warp loads 32 consecutive
// particles; consecutive lanes whose particles share a stencil base form a run;
// for each run, lane j < 27 owns stencil node j, sums the run's contributions in
// registers (particle data broadcast from shared memory) and issues one atomic
// per field. With particles ordered by cell this turns 27 atomics per particle
// into 27 per run of ~tens of particles, and any order stays correct.
//
// The active node box (min/max stencil node of the current particles) bounds
// every dense grid pass; the grid passes leave the scatter fields zeroed behind
// them, so no dense memset is needed between substeps.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdio>
#include <type_traits>
#include <utility>
#include <vector>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"
#include "bk_mlp.cuh"
#include "bk_profile.h"

using namespace bk;

namespace {

constexpr int kThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Kernel-side copy of the parameters (plain values only).
struct Params {
    int64_t n, pitch;
    int R, bc;
    float origin[3], dx, dt, gravity[3];
    int material;
    DingParamsDev ding;
    int transport, gas, settling;
    float oven, tray, tray_transfer, surface_loss, water_density, latent;
    int water_enabled;
    float conductivity, diffusivity, s0, water_stress;
    float ambient, density, elastic_modulus, cfl, peak, width;
    int keep_fields;
    int prescattered, prescatter_next, prescatter_stale;
    int32_t* status;
};

Params to_params(const BkSubstepParams& p) {
    Params k;
    k.n = p.n; k.pitch = p.pitch; k.R = p.resolution; k.bc = p.boundary_cells;
    for (int a = 0; a < 3; ++a) { k.origin[a] = p.origin[a]; k.gravity[a] = p.gravity[a]; }
    k.dx = p.spacing; k.dt = p.time_step;
    k.material = p.material;
    const BkDingParams& d = p.ding;
    k.ding.coupled_porosity = d.coupled_porosity; k.ding.temperature_enabled = d.temperature_enabled;
    k.ding.mu = d.shear_modulus; k.ding.lam = d.lame_lambda; k.ding.yield_stress = d.yield_stress;
    k.ding.initial_porosity = d.initial_porosity; k.ding.dt = d.time_step;
    for (int i = 0; i < 4; ++i) {
        k.ding.knots[i] = d.temperature_knots[i];
        k.ding.yield_factors[i] = d.yield_factors[i];
        k.ding.viscosity_factors[i] = d.viscosity_factors[i];
    }
    k.transport = p.transport; k.gas = p.gas; k.settling = p.settling;
    k.oven = p.scalar.oven_temperature; k.tray = p.scalar.tray_temperature;
    k.tray_transfer = p.scalar.tray_transfer; k.surface_loss = p.scalar.surface_loss;
    k.water_density = p.scalar.water_density; k.latent = p.scalar.latent_heat;
    k.water_enabled = p.scalar.water_enabled;
    k.conductivity = p.conductivity; k.diffusivity = p.diffusivity; k.s0 = p.initial_saturation;
    k.water_stress = p.water_stress;
    k.ambient = p.gas_ambient_pressure; k.density = p.density; k.elastic_modulus = p.elastic_modulus;
    k.cfl = p.cfl_limit; k.peak = p.gas_peak; k.width = p.gas_width;
    k.keep_fields = p.keep_transport_fields;
    k.prescattered = p.transport_prescattered;
    k.prescatter_next = p.transport_prescatter_next;
    k.prescatter_stale = p.transport_prescatter_stale;
    k.status = p.status;
    return k;
}

// The configuration of the loaf and dough bodies: Ding with temperature-dependent parameters, gas
// with the coupled porosity solve, thermal-water transport, no per-particle diagnostics and no
// harvest. The particle kernels have an instance for it in which these flags are compile-time
// constants, so the branches of the other configurations fold away (same arithmetic, less code).
bool loaf_mode(const BkSubstepParams& p, const BkDiagnostics& d) {
    return p.material == 1 && p.transport && p.gas && p.ding.coupled_porosity && p.ding.temperature_enabled &&
           !d.plastic_gradients && !d.return_residuals && !d.porosity_residuals &&
           !(p.surrogate && p.surrogate->samples);
}
__device__ __forceinline__ void fix_loaf_mode(Params& P) {
    P.material = 1;
    P.transport = 1;
    P.gas = 1;
    P.ding.coupled_porosity = 1;
    P.ding.temperature_enabled = 1;
}

struct GridPtrs {
    float4* pm;
    float4* v;
    double* f[7];
    double2* dTr;
    int* bounds;
};

GridPtrs grid_ptrs(const BkGrid& g) {
    GridPtrs r;
    r.pm = reinterpret_cast<float4*>(g.node_pm);
    r.v = reinterpret_cast<float4*>(g.node_v);
    for (int k = 0; k < 7; ++k) r.f[k] = g.fields[k];
    r.dTr = reinterpret_cast<double2*>(g.node_dT_ratio);
    r.bounds = g.bounds;
    return r;
}

// The block a kernel body runs as: its index among the blocks given to its simulator and their
// number. A plain launch gives one simulator the whole grid; a batched launch (below) splits its
// grid between the simulators of an instance table.
struct Slot {
    int block, blocks;
};
__device__ __forceinline__ Slot grid_slot() { return Slot{(int)blockIdx.x, (int)gridDim.x}; }

// Programmatic dependent launch between the kernels of a substep: each is launched with
// programmatic stream serialisation (launch_chained), so the launch of the next kernel and the
// placement of its blocks overlap the tail of the one before it. Every such kernel first waits
// until the kernel before it in the stream has completed and its memory is visible (which makes
// the chain transitive), then lets the next kernel launch; its blocks only take SM slots left free
// by blocks already running. A kernel without a programmatic predecessor returns from the wait at
// once.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The status of a launch_chained call, as check_launch reports a launch's.
int check_chained(cudaError_t e, const char* name) {
    if (e == cudaSuccess) return check_launch(name);
    cudaGetLastError();
    char msg[256];
    snprintf(msg, sizeof msg, "%s: %s", name, cudaGetErrorString(e));
    return fail(BK_ERR_LAUNCH, msg);
}

template <class... KArgs, class... Args>
cudaError_t launch_chained(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                           Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// How a kernel body takes its parameter structs: by value from a plain launch's parameter space
// (a reference to a kernel parameter would make the compiler copy it to local memory), by
// reference to the batched launch's shared-memory entry (a value copy would hold every field in
// registers).
template <class T, bool kRef>
using Arg = typename std::conditional<kRef, const T&, const T>::type;

// Stencil node j in 0..26 -> offsets (j / 9, (j / 3) % 3, j % 3), the reference's loop order.
__device__ __forceinline__ void node_offset(int j, int& ox, int& oy, int& oz) {
    ox = j / 9;
    oy = (j / 3) % 3;
    oz = j - 9 * ox - 3 * oy;
}


__device__ __forceinline__ long long pack_base(const int* b) {
    return ((long long)b[0] << 42) | ((long long)b[1] << 21) | (long long)b[2];
}

// Nodes a block may stage in shared memory before flushing them to the grid.
constexpr int kTileNodes = 512;

// Node box touched by one block's particles.
struct BlockBox {
    int lo[3], ext[3], count;  // count = 0: no valid particle in the block
    bool tiled;                // the box fits a shared-memory tile of kTileNodes
};

// Block-level min/max of valid stencil nodes; also widens the node box `bounds` ([0..2] lo, [3..5]
// hi) unless it is null. The box is tiled when it holds at most `tile_nodes` nodes. Every thread of the block must
// call this (it synchronises the block).
__device__ BlockBox block_box(int* bounds, bool valid, const int* b, int tile_nodes = kTileNodes) {
    __shared__ int s_box[6];
    if (threadIdx.x < 6) s_box[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int lo = __reduce_min_sync(kFull, valid ? b[a] : INT_MAX);
        int hi = __reduce_max_sync(kFull, valid ? b[a] + 2 : INT_MIN);
        if ((threadIdx.x & 31) == 0 && lo != INT_MAX) {
            atomicMin(&s_box[a], lo);
            atomicMax(&s_box[3 + a], hi);
        }
    }
    __syncthreads();
    BlockBox bb;
    bb.count = 0;
    bb.tiled = true;
    if (s_box[0] != INT_MAX) {
        long long count = 1;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bb.lo[a] = s_box[a];
            bb.ext[a] = s_box[3 + a] - s_box[a] + 1;
            count *= bb.ext[a];
        }
        bb.tiled = count <= tile_nodes;
        bb.count = bb.tiled ? (int)count : 0;
        if (bounds != nullptr && threadIdx.x < 3) {
            // The shared box only widens (min of lo, max of hi), so a value read through L2 that is
            // older than the current one is never narrower: a block whose box lies inside it
            // skips the atomics, and thousands of blocks stop contending for six addresses.
            const int t = threadIdx.x;
            if (s_box[t] < __ldcg(bounds + t)) atomicMin(bounds + t, s_box[t]);
            if (s_box[3 + t] > __ldcg(bounds + 3 + t)) atomicMax(bounds + 3 + t, s_box[3 + t]);
        }
    }
    return bb;
}

__device__ __forceinline__ int tile_index(const BlockBox& bb, int x, int y, int z) {
    return ((x - bb.lo[0]) * bb.ext[1] + (y - bb.lo[1])) * bb.ext[2] + (z - bb.lo[2]);
}

__device__ __forceinline__ int64_t tile_node(const BlockBox& bb, int t, int R) {
    int z = t % bb.ext[2];
    int y = (t / bb.ext[2]) % bb.ext[1];
    int x = t / (bb.ext[2] * bb.ext[1]);
    return node_index(bb.lo[0] + x, bb.lo[1] + y, bb.lo[2] + z, R);
}

// ------------------------------------------------------------------ surface
// geometry/mesh_tracking.py:13-38 restricted to the vertices of boundary faces. A vertex of a
// coarse mesh binds thousands of particles: one block of kBlock = 128 or 256 threads per vertex
// keeps enough gathers in flight. A vertex of a fine mesh binds tens: kBlock = 32 then means one
// warp per vertex, kVertexWarps vertices to a block.
constexpr int kVertexWarps = 8;

// Blocks of the surface vertex launch for `vertices` vertices at block size `threads`.
inline unsigned vertex_launch_blocks(int64_t vertices, int threads) {
    return (unsigned)(threads == 32 ? (vertices + kVertexWarps - 1) / kVertexWarps : vertices);
}
inline int vertex_launch_threads(int threads) { return threads == 32 ? 32 * kVertexWarps : threads; }

template <int kBlock, bool kRef = false>
__device__ __forceinline__ void surface_vertices_body(Arg<Params, kRef> P, const float* __restrict__ x,
                                                      const float* __restrict__ F, Arg<BkSurface, kRef> sf, Slot sl) {
    if constexpr (kBlock == 32) {
        const int64_t k = (int64_t)sl.block * kVertexWarps + (threadIdx.x >> 5);
        if (k >= sf.vertex_count) return;  // whole warps
        const int vid = sf.vertex_ids[k];
        const float v = vertex_warp(sf.binding_offsets, sf.binding_particles, sf.binding_weights,
                                    sf.reference_offsets, sf.binding_pitch, sf.reference_vertices, sf.vertex_pitch, x,
                                    F, P.pitch, vid);
        const int lane = threadIdx.x & 31;
        if (lane < 3) sf.vertices[lane * sf.vertex_pitch + vid] = v;
    } else {
        const int vid = sf.vertex_ids[sl.block];
        const float v = vertex_block<kBlock>(sf.binding_offsets, sf.binding_particles, sf.binding_weights,
                                               sf.reference_offsets, sf.binding_pitch, sf.reference_vertices,
                                               sf.vertex_pitch, x, F, P.pitch, vid);
        if (threadIdx.x < 3) sf.vertices[threadIdx.x * sf.vertex_pitch + vid] = v;
    }
}

template <int kBlock>
__global__ void __launch_bounds__(kBlock == 32 ? 32 * kVertexWarps : kBlock) k_surface_vertices(Params P, const float* __restrict__ x,
                                                          const float* __restrict__ F, BkSurface sf) {
    pdl_enter();
    surface_vertices_body<kBlock>(P, x, F, sf, grid_slot());
}

// ------------------------------------------------------- surface terms
// physics/thermal_water.py:77-92 (face areas, tray contact) and the surface terms of :108-122 for
// the face-owning particles, in two layouts chosen by how many particles own faces:
// * few owners, each with several faces (a coarse voxel mesh: about 3k owners of a 1M-particle
//   loaf): one warp per owner; lane 0 sums the owner's faces in order, every lane forms the rates,
//   lane j < 27 adds stencil node j's share (27 atomics in parallel);
// * many owners (a fine tetrahedral mesh: about a third of a dough ball's particles own faces): one
//   thread per owner, the node shares summed per stencil run and per block tile like the transport
//   scatter, so the 81 float64 atomics per owner become a few per node and block.
// With accumulators set in `sf`, the owner's water-loss and heat-exchange accumulators also advance
// by one substep (thermal_water.py:225-226), which bk_surface_accumulate does otherwise.
constexpr int kOwnerThreads = 128;

// Exposed and tray-contact areas of owner o's faces, summed in face order.
template <class SF>
__device__ __forceinline__ void owner_areas(const SF& sf, int64_t o, double& exposed, double& contact) {
    const int64_t vp = sf.vertex_pitch;
    exposed = 0.0;
    contact = 0.0;
    for (int f = sf.owner_face_offsets[o]; f < sf.owner_face_offsets[o + 1]; ++f) {
        double q[3][3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int vid = sf.faces[3 * f + k];
#pragma unroll
            for (int a = 0; a < 3; ++a) q[k][a] = (double)sf.vertices[a * vp + vid];
        }
        double e1[3] = {q[1][0] - q[0][0], q[1][1] - q[0][1], q[1][2] - q[0][2]};
        double e2[3] = {q[2][0] - q[0][0], q[2][1] - q[0][1], q[2][2] - q[0][2]};
        double nr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        double len = sqrt(nr[0] * nr[0] + nr[1] * nr[1] + nr[2] * nr[2]);
        double area = 0.5 * len;
        double cy = (q[0][1] + q[1][1] + q[2][1]) / 3.0;
        if (cy <= (double)(sf.floor_height + sf.contact_distance) && nr[1] < -0.2 * len) contact += area;
        else exposed += area;
    }
}

// Heat, loss and exchange rates of owner particle p from its areas; rate[0..2].
template <class PP, class ST, class CS>
__device__ __forceinline__ void owner_rates(const PP& P, const ST& in, const CS& cst, int p, double exposed,
                                            double contact, double* rate) {
    const int64_t pitch = P.pitch;
    double vol = (double)cst.volume[p] * (double)det3(load_m3(in.F, p, pitch));
    double T = in.temperature[p], W = in.water[p];
    double sat = W / ((double)P.water_density * vol);
    double loss = 0.0;
    if (P.water_enabled) loss = (double)P.surface_loss * T * sat * exposed;
    double h = (double)cst.heat_parameter[0];
    double heat = h * exposed * ((double)P.oven - T) + (double)P.tray_transfer * contact * ((double)P.tray - T)
                - (double)P.latent * loss;
    double exch = h * exposed + (double)P.tray_transfer * contact;
    if (P.water_enabled) exch += (double)(P.latent * P.surface_loss) * sat * exposed;
    rate[0] = heat;
    rate[1] = loss;
    rate[2] = exch;
}

// Stores owner o's rates and advances its accumulators when `sf` names them.
template <class SF>
__device__ __forceinline__ void owner_store(const SF& sf, int64_t o, int p, const double* rate) {
    sf.owner_heat[o] = rate[0];
    sf.owner_loss[o] = rate[1];
    if (sf.accumulate_water_losses) {
        sf.accumulate_water_losses[p] += (double)sf.accumulate_time_step * rate[1];
        sf.accumulate_heat_exchanges[p] += (double)sf.accumulate_time_step * rate[0];
    }
}

template <bool kRef = false>
__device__ __forceinline__ void surface_owners_warp_body(Arg<Params, kRef> P, Arg<BkState, kRef> in,
                                                         Arg<BkConstants, kRef> cst, Arg<BkSurface, kRef> sf,
                                                         Arg<GridPtrs, kRef> g, int32_t* sim_flags, Slot sl) {
    const int lane = threadIdx.x & 31;
    const int64_t o = (sl.block * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (o >= sf.owner_count) return;  // whole warps
    const int p = sf.owners[o];
    double exposed = 0.0, contact = 0.0;
    if (lane == 0) owner_areas(sf, o, exposed, contact);
    exposed = __shfl_sync(kFull, exposed, 0);
    contact = __shfl_sync(kFull, contact, 0);
    double rate[3];
    owner_rates(P, in, cst, p, exposed, contact, rate);
    if (lane == 0) owner_store(sf, o, p, rate);
    Stencil st = make_stencil(load_v3(in.x, p, P.pitch), P.origin, P.dx, P.R);
    if (!st.valid) {
        if (lane == 0) set_flag(sim_flags, 1);
        return;
    }
    if (lane < 27) {
        int ox, oy, oz;
        node_offset(lane, ox, oy, oz);
        double w = (double)(st.w[0][ox] * st.w[1][oy] * st.w[2][oz]);
        int64_t node = node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R);
        atomicAdd(g.f[4] + node, w * rate[0]);
        atomicAdd(g.f[5] + node, w * rate[1]);
        atomicAdd(g.f[6] + node, w * rate[2]);
    }
}

// ---------------------------------------------------------- transport P2G
// physics/thermal_water.py:108-137 (volume, capacity, energy, water), warp-cooperative per stencil run.
// The block routine scatters its threads' particles; each thread passes its stencil, whether it is
// valid, and its four values (V0 det F, capacity, capacity T, W). Every thread of the block calls it.
// The run sums are float64, as the reference's float64 atomics: float32 partial sums moved the
// node temperature E/C by ~3e-5 K, harmless to the trajectory but enough to make finite
// differences of the loss in the initial temperatures disagree with the adjoint by several percent.
// The routine is shared with the surface terms (heat, loss and exchange of the face owners into
// node fields 4..6): kF fields starting at node field kFirst, values of invalid threads ignored.
// Stencil weights of the block's particles, in one of two forms:
// * kNodeWeights: each particle's 27 weights (w_x w_y) w_z, formed once by its own thread as the
//   reference rounds them, in node-major rows of kT + 1 floats; lane j of a run reads row j at the
//   particle's column, one conflict-free load in place of three loads and two multiplies per node;
// * otherwise the nine axis weights per particle (3 loads and 2 multiplies per node), a third of
//   the space: the form of the scatter inside the G2P kernel, whose eight blocks per SM leave the
//   rest of the SM's shared memory to L1 for its spilled registers (the 27-weight rows there made
//   that kernel 4 us slower at 1M particles while the standalone scatter gained 4 us).
template <int kT, bool kNodeWeights>
struct ScatterWeights;
template <int kT>
struct ScatterWeights<kT, true> {
    float w[27][kT + 1];
    __device__ __forceinline__ void put(int tid, bool valid, const Stencil& st) {
#pragma unroll
        for (int ox = 0; ox < 3; ++ox)
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float wxy = st.w[0][ox] * st.w[1][oy];
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) w[9 * ox + 3 * oy + oz][tid] = valid ? wxy * st.w[2][oz] : 0.f;
            }
    }
    // weight of node (ox, oy, oz) = lane j for particle k
    __device__ __forceinline__ float get(int k, int j, int, int, int) const { return w[j][k]; }
};
template <int kT>
struct ScatterWeights<kT, false> {
    float w[kT][9];
    __device__ __forceinline__ void put(int tid, bool valid, const Stencil& st) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int o = 0; o < 3; ++o) w[tid][3 * a + o] = valid ? st.w[a][o] : 0.f;
    }
    __device__ __forceinline__ float get(int k, int, int ox, int oy, int oz) const {
        return w[k][ox] * w[k][3 + oy] * w[k][6 + oz];
    }
};

template <int kT, int kTile, int kF = 4, bool kNodeWeights = true>
struct TransportTile {
    ScatterWeights<kT, kNodeWeights> w;
    double val[kT][kF];
    double tile[kF][kTile];
};

template <int kT, int kTile, int kF = 4, int kFirst = 0, bool kNodeWeights = true>
__device__ void transport_scatter_block(TransportTile<kT, kTile, kF, kNodeWeights>& sm, const Params& P, const GridPtrs& g, int* box,
                                        bool valid, const Stencil& st, const double* val) {
    static_assert(kF >= 1 && kF <= 4 && kFirst + kF <= 7, "node fields 0..6, at most four at a time");
    const int tid = threadIdx.x, lane = tid & 31;
#pragma unroll
    for (int f = 0; f < kF; ++f) sm.val[tid][f] = valid ? val[f] : 0.0;
    sm.w.put(tid, valid, st);
    const BlockBox bb = block_box(box, valid, st.b, kTile);  // synchronises the block
    for (int t = tid; t < bb.count; t += kT)
#pragma unroll
        for (int f = 0; f < kF; ++f) sm.tile[f][t] = 0.0;
    __syncthreads();
    long long key = valid ? pack_base(st.b) : -1;
    long long prev = __shfl_up_sync(kFull, key, 1);
    unsigned starts = __ballot_sync(kFull, valid && (lane == 0 || prev != key));
    const int warp_base = tid & ~31;
    int ox, oy, oz;
    node_offset(lane < 27 ? lane : 0, ox, oy, oz);
    while (starts) {
        int s = __ffs(starts) - 1;
        starts &= starts - 1;
        int e = starts ? __ffs(starts) - 1 : 32;
        int b0 = __shfl_sync(kFull, st.b[0], s), b1 = __shfl_sync(kFull, st.b[1], s), b2 = __shfl_sync(kFull, st.b[2], s);
        if (lane < 27) {
            // Even and odd particles of the run into separate sums: two independent chains of
            // float64 multiply-adds per field, so consecutive particles' loads and conversions overlap.
            double acc[kF], acc_odd[kF];
#pragma unroll
            for (int f = 0; f < kF; ++f) acc[f] = acc_odd[f] = 0.0;
            int k = warp_base + s;
            const int k_end = warp_base + e;
            for (; k + 1 < k_end; k += 2) {
                const double w0 = (double)sm.w.get(k, lane, ox, oy, oz);
                const double w1 = (double)sm.w.get(k + 1, lane, ox, oy, oz);
#pragma unroll
                for (int f = 0; f < kF; ++f) {
                    acc[f] = fma(w0, sm.val[k][f], acc[f]);
                    acc_odd[f] = fma(w1, sm.val[k + 1][f], acc_odd[f]);
                }
            }
            if (k < k_end) {
                const double w0 = (double)sm.w.get(k, lane, ox, oy, oz);
#pragma unroll
                for (int f = 0; f < kF; ++f) acc[f] = fma(w0, sm.val[k][f], acc[f]);
            }
#pragma unroll
            for (int f = 0; f < kF; ++f) acc[f] += acc_odd[f];
            if (bb.tiled) {
                int t = tile_index(bb, b0 + ox, b1 + oy, b2 + oz);
#pragma unroll
                for (int f = 0; f < kF; ++f) atomicAdd(&sm.tile[f][t], acc[f]);
            } else {
                int64_t node = node_index(b0 + ox, b1 + oy, b2 + oz, P.R);
#pragma unroll
                for (int f = 0; f < kF; ++f) atomicAdd(g.f[kFirst + f] + node, acc[f]);
            }
        }
    }
    __syncthreads();
    for (int t = tid; t < bb.count; t += kT) {
        bool empty = true;
#pragma unroll
        for (int f = 0; f < kF; ++f) empty = empty && sm.tile[f][t] == 0.0;
        if (empty) continue;
        int64_t node = tile_node(bb, t, P.R);
#pragma unroll
        for (int f = 0; f < kF; ++f) atomicAdd(g.f[kFirst + f] + node, sm.tile[f][t]);
    }
}

template <bool kRef = false>
__device__ __forceinline__ void surface_owners_tile_body(Arg<Params, kRef> P, Arg<BkState, kRef> in,
                                                         Arg<BkConstants, kRef> cst, Arg<BkSurface, kRef> sf,
                                                         Arg<GridPtrs, kRef> g, int32_t* sim_flags, Slot sl) {
    __shared__ TransportTile<kOwnerThreads, kTileNodes, 3> sm;
    const int64_t o = sl.block * (int64_t)kOwnerThreads + threadIdx.x;
    bool valid = false;
    Stencil st;
    st.b[0] = st.b[1] = st.b[2] = 0;
    double rate[3] = {0.0, 0.0, 0.0};
    if (o < sf.owner_count) {
        const int p = sf.owners[o];
        double exposed, contact;
        owner_areas(sf, o, exposed, contact);
        owner_rates(P, in, cst, p, exposed, contact, rate);
        owner_store(sf, o, p, rate);
        st = make_stencil(load_v3(in.x, p, P.pitch), P.origin, P.dx, P.R);
        valid = st.valid;
        if (!valid) set_flag(sim_flags, 1);
    }
    // the owners' nodes lie inside the particles' transport box: no box to widen
    transport_scatter_block<kOwnerThreads, kTileNodes, 3, 4>(sm, P, g, nullptr, valid, st, rate);
}

// Many owners take the tiled form (one thread each), few the warp form (one warp each).
template <bool kRef = false>
__device__ __forceinline__ void surface_owners_body(Arg<Params, kRef> P, Arg<BkState, kRef> in, Arg<BkConstants, kRef> cst,
                                                    Arg<BkSurface, kRef> sf, Arg<GridPtrs, kRef> g, int32_t* sim_flags,
                                                    bool tiled, Slot sl) {
    if (tiled) surface_owners_tile_body<kRef>(P, in, cst, sf, g, sim_flags, sl);
    else surface_owners_warp_body<kRef>(P, in, cst, sf, g, sim_flags, sl);
}

// Whether a body with `owners` face owners among `n` particles takes the tiled form, and its blocks.
inline bool owners_tiled(int64_t owners, int64_t n) { return owners * 16 >= n; }
inline unsigned owner_blocks(int64_t owners, int64_t n) {
    const int64_t threads = owners_tiled(owners, n) ? owners : owners * 32;
    return (unsigned)((threads + kOwnerThreads - 1) / kOwnerThreads);
}

__global__ void __launch_bounds__(kOwnerThreads) k_surface_owners(Params P, BkState in, BkConstants cst, BkSurface sf,
                                                                 GridPtrs g, int32_t* sim_flags, int tiled) {
    pdl_enter();
    surface_owners_body(P, in, cst, sf, g, sim_flags, tiled != 0, grid_slot());
}

// 256 nodes: the 27 weight rows of 256 particles leave room for no larger tile in 48 KB of static shared memory.
using ScatterTile = TransportTile<kThreads, 256>;

template <bool kRef = false>
__device__ __forceinline__ void transport_scatter_body(Arg<Params, kRef> P, Arg<BkState, kRef> in,
                                                       Arg<BkConstants, kRef> cst, Arg<GridPtrs, kRef> g, int32_t* sim_flags,
                                                       Slot sl) {
    // Shared memory is declared in the bodies, not passed in: through a reference the compiler may
    // not see that it is shared memory and issue generic loads, stores and atomics.
    __shared__ ScatterTile sm;
    const int64_t i = sl.block * (int64_t)kThreads + threadIdx.x;
    const int64_t pitch = P.pitch;
    bool valid = false;
    Stencil st;
    st.b[0] = st.b[1] = st.b[2] = 0;
    double val[4] = {0.0, 0.0, 0.0, 0.0};
    if (i < P.n) {
        st = make_stencil(load_v3(in.x, i, pitch), P.origin, P.dx, P.R);
        valid = st.valid;
        if (!valid) set_flag(sim_flags, 1);
    }
    if (valid) {
        double cap = cst.capacity[i];
        val[0] = (double)cst.volume[i] * (double)det3(load_m3(in.F, i, pitch));
        val[1] = cap;
        val[2] = cap * in.temperature[i];
        val[3] = in.water[i];
    }
    transport_scatter_block<kThreads, 256>(sm, P, g, g.bounds, valid, st, val);
}

__global__ void __launch_bounds__(kThreads) k_transport_scatter(Params P, BkState in, BkConstants cst, GridPtrs g,
                                                               int32_t* sim_flags) {
    pdl_enter();
    transport_scatter_body(P, in, cst, g, sim_flags, grid_slot());
}

// ------------------------------------------------------------ grid passes
// Node box [lo, hi] of `bounds` clipped to the grid; false when it is empty. The empty box is
// stored as lo = INT_MAX, hi = INT_MIN, so emptiness is tested before any subtraction.
__device__ __forceinline__ bool box_of(const int* bounds, int R, int lo[3], int ext[3], int64_t& count) {
    count = 1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int l = bounds[a], h = bounds[3 + a];
        if (l > h) return false;
        l = max(l, 0);
        h = min(h, R - 1);
        if (l > h) return false;
        lo[a] = l;
        ext[a] = h - l + 1;
        count *= ext[a];
    }
    return true;
}

// physics/thermal_water.py:140-190: node temperature/saturation (GridFields) and the 7-point flux
// (DiffuseGrid) over the active box, tiled through shared memory. A block takes a tile of
// kDiffX x kDiffY x kDiffZ nodes (z fastest, one warp per z row) and first stages the tile plus a
// one-node halo: for each staged node with capacity it forms T = E / C and s = W / (rho_w V) once,
// keeping V, T, s and the capacity test in shared memory. The six-neighbour stencil then reads only
// shared memory, so each node's fields are read from L2/HBM about (1 + halo) times instead of seven,
// and each node's two float64 divisions run once instead of once per neighbour.
constexpr int kDiffX = 2, kDiffY = 4, kDiffZ = 32;
constexpr int kDiffThreads = kDiffX * kDiffY * kDiffZ;
constexpr int kHaloX = kDiffX + 2, kHaloY = kDiffY + 2, kHaloZ = kDiffZ + 2;
constexpr int kHaloNodes = kHaloX * kHaloY * kHaloZ;

struct DiffuseSmem {
    double V[kHaloNodes], T[kHaloNodes], S[kHaloNodes];
    unsigned char ok[kHaloNodes];
};

template <bool kRef = false>
__device__ __forceinline__ void diffuse_body(Arg<Params, kRef> P, Arg<GridPtrs, kRef> g, int32_t* errors,
                                             Slot sl) {
    __shared__ DiffuseSmem sm;
    double* s_V = sm.V;
    double* s_T = sm.T;
    double* s_S = sm.S;
    unsigned char* s_ok = sm.ok;
    int lo[3], ext[3];
    int64_t count;
    // The node box of the transport fields: built by this substep's scalar P2G, or by the previous
    // substep's G2P when it scattered them ahead.
    if (!box_of(P.prescattered ? g.bounds + 12 : g.bounds, P.R, lo, ext, count)) return;
    const int R = P.R;
    const double rho_w = (double)P.water_density;
    const double cell = (double)(P.dx * P.dx * P.dx);
    const double kc = (double)(P.conductivity * P.dx);
    const double kw = (double)(P.diffusivity * P.water_density * P.dx);
    const double dt = (double)P.dt;
    const int tiles_z = (ext[2] + kDiffZ - 1) / kDiffZ, tiles_y = (ext[1] + kDiffY - 1) / kDiffY;
    const int tiles_x = (ext[0] + kDiffX - 1) / kDiffX;
    const int tiles = tiles_x * tiles_y * tiles_z;
    const int tid = threadIdx.x;
    const int tz = tid % kDiffZ, ty = (tid / kDiffZ) % kDiffY, tx = tid / (kDiffZ * kDiffY);
    for (int tile = sl.block; tile < tiles; tile += sl.blocks) {
        const int t0[3] = {lo[0] + (tile / (tiles_z * tiles_y)) * kDiffX, lo[1] + ((tile / tiles_z) % tiles_y) * kDiffY,
                           lo[2] + (tile % tiles_z) * kDiffZ};
        // Stage the tile and its halo (nodes outside the grid are marked empty, like the reference's
        // range test; nodes outside the box but inside the grid hold zero fields).
        for (int h = tid; h < kHaloNodes; h += kDiffThreads) {
            const int hz = h % kHaloZ, hy = (h / kHaloZ) % kHaloY, hx = h / (kHaloZ * kHaloY);
            const int c0 = t0[0] + hx - 1, c1 = t0[1] + hy - 1, c2 = t0[2] + hz - 1;
            bool ok = c0 >= 0 && c0 < R && c1 >= 0 && c1 < R && c2 >= 0 && c2 < R;
            double V = 0.0, T = 0.0, S = 0.0;
            if (ok) {
                const int64_t j = node_index(c0, c1, c2, R);
                const double cj = g.f[1][j];
                ok = cj > 0.0;
                if (ok) {
                    V = g.f[0][j];
                    T = g.f[2][j] / cj;
                    S = g.f[3][j] / (rho_w * V);
                }
            }
            s_V[h] = V;
            s_T[h] = T;
            s_S[h] = S;
            s_ok[h] = ok;
        }
        __syncthreads();
        const int c[3] = {t0[0] + tx, t0[1] + ty, t0[2] + tz};
        const int h = ((tx + 1) * kHaloY + (ty + 1)) * kHaloZ + (tz + 1);
        if (c[0] < lo[0] + ext[0] && c[1] < lo[1] + ext[1] && c[2] < lo[2] + ext[2]) {
            const int64_t i = node_index(c[0], c[1], c[2], R);
            if (!s_ok[h]) {
                g.dTr[i] = make_double2(0.0, 0.0);
            } else {
                const double ci = g.f[1][i], Wi = g.f[3][i];
                const double vi = s_V[h], Ti = s_T[h], si = s_S[h];
                double heat_rate = g.f[4][i], water_rate = -g.f[5][i], heat_diag = g.f[6][i], water_diag = 0.0;
                const int stride[3] = {kHaloY * kHaloZ, kHaloZ, 1};
#pragma unroll
                for (int axis = 0; axis < 3; ++axis)
#pragma unroll
                    for (int side = 0; side < 2; ++side) {
                        const int hj = h + (2 * side - 1) * stride[axis];
                        if (!s_ok[hj]) continue;
                        const double vj = s_V[hj], Tj = s_T[hj];
                        const double fill = 2.0 * vi * vj / (vi + vj) / cell;
                        const double hc = kc * fill;
                        heat_rate += hc * (Tj - Ti);
                        heat_diag += hc;
                        if (P.water_enabled) {
                            const double sj = s_S[hj];
                            const double mob = kw * fill * 0.5 * (Ti + Tj) * 0.5 * (si + sj);
                            water_rate += mob * (sj - si);
                            water_diag += mob / (rho_w * vi);
                        }
                    }
                if (dt * heat_diag > ci) set_flag(errors, 0);
                const double change = dt * water_rate;
                if (Wi + change < 0.0 || dt * water_diag > 1.0) set_flag(errors, 1);
                const double dT = dt * heat_rate / ci;
                g.dTr[i] = make_double2(dT, Wi > 0.0 ? change / Wi : 0.0);
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kDiffThreads) k_diffuse(Params P, GridPtrs g, int32_t* errors) {
    pdl_enter();
    diffuse_body(P, g, errors, grid_slot());
}

// Fields scattered ahead for a substep that runs its own scalar P2G instead (the state may have
// changed in between): zero the volume, capacity, energy and water fields over their box.
template <bool kRef = false>
__device__ __forceinline__ void clear_prescatter_body(Arg<Params, kRef> P, Arg<GridPtrs, kRef> g, Slot sl) {
    int lo[3], ext[3];
    int64_t count;
    if (!box_of(g.bounds + 12, P.R, lo, ext, count)) return;
    for (int64_t t = sl.block * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)sl.blocks * blockDim.x) {
        int c2 = lo[2] + (int)(t % ext[2]);
        int c1 = lo[1] + (int)((t / ext[2]) % ext[1]);
        int c0 = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        int64_t i = node_index(c0, c1, c2, P.R);
#pragma unroll
        for (int k = 0; k < 4; ++k) g.f[k][i] = 0.0;
    }
}

__global__ void k_clear_prescatter(Params P, GridPtrs g) {
    pdl_enter();
    clear_prescatter_body(P, g, grid_slot());
}

// GridState.Clear (physics/grid.py:14-17) restricted to the previous substep's active box, the only
// nodes holding nonzero momentum, mass or velocity; the grid of the last substep stays readable
// until the next one starts.
template <bool kRef = false>
__device__ __forceinline__ void clear_previous_body(Arg<Params, kRef> P, Arg<GridPtrs, kRef> g, Slot sl) {
    int lo[3], ext[3];
    int64_t count;
    if (!box_of(g.bounds + 6, P.R, lo, ext, count)) return;
    for (int64_t t = sl.block * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)sl.blocks * blockDim.x) {
        int c2 = lo[2] + (int)(t % ext[2]);
        int c1 = lo[1] + (int)((t / ext[2]) % ext[1]);
        int c0 = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        int64_t i = node_index(c0, c1, c2, P.R);
        g.pm[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        g.v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

__global__ void k_clear_previous(Params P, GridPtrs g) {
    pdl_enter();
    clear_previous_body(P, g, grid_slot());
}

// physics/grid.py:20-38 over the active box; clears the transport scatter fields behind it.
template <bool kRef = false>
__device__ __forceinline__ void grid_update_body(Arg<Params, kRef> P, Arg<GridPtrs, kRef> g, Slot sl) {
    int lo[3], ext[3];
    int64_t count;
    // The G2P that follows builds the next substep's transport box in bounds[12..17]: restart it
    // empty (this substep's diffusion, its only reader, has finished; no block here reads it).
    if (P.prescatter_next && sl.block == 0 && threadIdx.x < 6) g.bounds[12 + threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
    if (!box_of(g.bounds, P.R, lo, ext, count)) return;
    const int R = P.R, bc = P.bc;
    for (int64_t t = sl.block * (int64_t)blockDim.x + threadIdx.x; t < count; t += (int64_t)sl.blocks * blockDim.x) {
        int c[3];
        c[2] = lo[2] + (int)(t % ext[2]);
        c[1] = lo[1] + (int)((t / ext[2]) % ext[1]);
        c[0] = lo[0] + (int)(t / ((int64_t)ext[2] * ext[1]));
        int64_t i = node_index(c[0], c[1], c[2], R);
        float4 pm = g.pm[i];
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (pm.w > 0.0f) {
            float vel[3] = {pm.x / pm.w + P.dt * P.gravity[0], pm.y / pm.w + P.dt * P.gravity[1],
                            pm.z / pm.w + P.dt * P.gravity[2]};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                if (c[a] < bc && vel[a] < 0.0f) vel[a] = 0.0f;
                if (c[a] >= R - bc && vel[a] > 0.0f) vel[a] = 0.0f;
            }
            out = make_float4(vel[0], vel[1], vel[2], 0.f);
        }
        g.v[i] = out;
        if (P.transport && !P.keep_fields) {
#pragma unroll
            for (int k = 0; k < 7; ++k) g.f[k][i] = 0.0;
        }
    }
}

__global__ void k_grid_update(Params P, GridPtrs g) {
    pdl_enter();
    grid_update_body(P, g, grid_slot());
}

// ------------------------------------------------------------- fused P2G
// Scalar G2P (thermal_water.py:206-229), local gas source (:238-245), gas stress (gas.py:16-35),
// water stress (thermal_water.py:248-253) and momentum P2G (transfer.py:47-70) for one particle
// per thread, then the warp-cooperative momentum scatter.
// One particle's scatter record: its 27 stencil weights (w_x w_y) w_z, formed once by its own
// thread, in node-major rows of kThreads + 1 floats (lane j of a run reads row j at the particle's
// column: one conflict-free load per node in place of three loads and two multiplies), and
// {m q0 q1 q2} {A0 A1 A2 A3} {A4 A5 A6 A7} read as 128-bit broadcasts plus A8.
// The staged form first copies the block's particle planes (x, v, C, F and, for Ding, tau: 33
// planes of 256 floats) into shared memory with bulk copies (cp.async.bulk, the TMA engine's 1-D
// copy) issued by one thread and counted on an mbarrier, so the loads of a block are in flight
// together and each thread then reads its particle's 33 values from shared memory; the scatter
// records reuse that space once every thread has read it.
// A full block (256 particles) also stages its per-particle scalars: temperature, water, dry mass
// and gas content (float64), reference volume, gas source rate and porosity (float32), those the
// substep reads; the last, partial block loads them directly (the arrays need not extend past n).
constexpr int kP2GPlanes = 33;
struct P2GSmem {
    union {
        struct {
            float planes[kP2GPlanes][kThreads];  // x 0-2 (unused: x is read directly), v 3-5, C 6-14, F 15-23, tau 24-32
            double d[4][kThreads];               // temperature, water, dry mass, gas moles
            float f[3][kThreads];                // reference volume, gas source rate, porosity
        } in;
        struct {
            float4 val[kThreads][3];
            float a8[kThreads];
            float w[27][kThreads + 1];
        } rec;
    };
    float4 tile[kTileNodes];
    unsigned long long mbar;
};
// Above the 48 KB of static shared memory: the kernels take it as dynamic shared memory, opted in
// per device before their first launch there.
constexpr size_t kP2GSmemBytes = sizeof(P2GSmem);

// Which per-particle scalars a full P2G block stages (bit k of d[k], bit 4 + k of f[k]).
__host__ __device__ inline unsigned p2g_staged_scalars(int transport, int gas, int material, int rate_per_particle) {
    unsigned m = 0;
    if (transport) m |= 1u | 2u | 4u | 16u;
    if (transport && gas) m |= 8u | (rate_per_particle ? 32u : 0u);
    if (material == 1 && gas) m |= 64u;
    return m;
}

// OR of the base addresses the bulk-staged P2G copies from (each must be 16-byte aligned).
inline uintptr_t p2g_stage_bases(const BkSubstepParams& p, const BkState& in, const BkConstants& c) {
    uintptr_t b = (uintptr_t)in.x | (uintptr_t)in.v | (uintptr_t)in.C | (uintptr_t)in.F |
                  (p.material == 1 ? (uintptr_t)in.tau : 0);
    const unsigned m = p2g_staged_scalars(p.transport, p.gas, p.material, c.gas_rate_per_particle);
    if (m & 1u) b |= (uintptr_t)in.temperature;
    if (m & 2u) b |= (uintptr_t)in.water;
    if (m & 4u) b |= (uintptr_t)c.dry_mass;
    if (m & 8u) b |= (uintptr_t)in.gas_moles;
    if (m & 16u) b |= (uintptr_t)c.volume;
    if (m & 32u) b |= (uintptr_t)c.gas_rate;
    if (m & 64u) b |= (uintptr_t)in.porosity;
    return b;
}

// Opts `kernel` into `bytes` of dynamic shared memory on the current device. Set on every launch:
// a host call without device work, and correct after a device reset or in another context.
int allow_smem(const void* kernel, size_t bytes, const char* what) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return check_launch(what);
    return 0;
}

namespace stage {
// Polls of a bulk copy's mbarrier before a block gives up (far beyond any copy's latency).
constexpr uint32_t kWaitPolls = 1u << 22;

__device__ __forceinline__ void arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// 1-D bulk copy global -> this CTA's shared memory, completing `bytes` on the mbarrier. Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void copy(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}
}  // namespace stage

// Four 256-thread blocks per SM (64 registers) measured faster than three at 77 registers.
template <bool kStaged, bool kRef = false>
__device__ __forceinline__ void p2g_body(Arg<Params, kRef> P, Arg<BkState, kRef> in, Arg<BkState, kRef> out,
                                         Arg<BkConstants, kRef> cst, Arg<GridPtrs, kRef> g, Arg<BkFlags, kRef> flags,
                                         float* max_residuals, Slot sl) {
    extern __shared__ __align__(16) unsigned char p2g_smem[];
    P2GSmem& sm = *reinterpret_cast<P2GSmem*>(p2g_smem);
    if (sl.block == 0 && threadIdx.x < 2) max_residuals[threadIdx.x] = 0.0f;
    const int tid = threadIdx.x, lane = tid & 31;
    const int64_t i = sl.block * (int64_t)kThreads + tid;
    const int64_t pitch = P.pitch;
    // Scalars this block reads from shared memory (full blocks of the staged form), by bit as in
    // p2g_staged_scalars; the others are loaded directly.
    const unsigned staged_scalars =
        kStaged && P.n - (int64_t)sl.block * kThreads >= kThreads
            ? p2g_staged_scalars(P.transport, P.gas, P.material, cst.gas_rate_per_particle) : 0u;
    // The particle's stencil and its scalar G2P of the diffused node fields (thermal_water.py:206-215)
    // read only x and the grid: the staged form runs them while its bulk copies are in flight.
    bool valid = false;
    Stencil st;
    st.b[0] = st.b[1] = st.b[2] = 0;
    double dTp = 0.0, ratio = 0.0;
    auto stencil_and_gather = [&]() {
        if (i < P.n) {
            st = make_stencil(load_v3(in.x, i, pitch), P.origin, P.dx, P.R);
            valid = st.valid;
            if (!valid) set_flag(flags.simulation, 1);
        }
        if (valid && P.transport) {
#pragma unroll
            for (int ox = 0; ox < 3; ++ox)
#pragma unroll
                for (int oy = 0; oy < 3; ++oy)
#pragma unroll
                    for (int oz = 0; oz < 3; ++oz) {
                        double w = (double)(st.w[0][ox] * st.w[1][oy] * st.w[2][oz]);
                        double2 d = __ldg(g.dTr + node_index(st.b[0] + ox, st.b[1] + oy, st.b[2] + oz, P.R));
                        dTp += w * d.x;
                        ratio += w * d.y;
                    }
        }
    };
    if constexpr (kStaged) {
        // Planes are pitch-long with a pitch that is a multiple of 4 and 16-byte aligned bases (the
        // host checks), so the block's range rounded up to 16 bytes stays inside each plane. The x
        // planes are not copied: x is read directly, before the wait.
        const uint32_t mbar = mlp::smem_addr(&sm.mbar);
        if (tid == 0) mlp::mbar_init(mbar, 1);
        __syncthreads();
        const int64_t start = (int64_t)sl.block * kThreads;
        if (tid == 0) {
            const int64_t count = P.n - start < kThreads ? P.n - start : kThreads;
            const uint32_t bytes = (uint32_t)((count * 4 + 15) & ~15ll);
            const int arrays = P.material == 1 ? 5 : 4;
            const float* src[5] = {in.x, in.v, in.C, in.F, in.tau};
            const int planes[5] = {3, 3, 9, 9, 9};
            const unsigned m = count == kThreads ? staged_scalars : 0u;
            uint32_t total = bytes * (uint32_t)(P.material == 1 ? kP2GPlanes - 3 : kP2GPlanes - 12);
#pragma unroll
            for (int k = 0; k < 7; ++k)
                if (m & (1u << k)) total += k < 4 ? kThreads * 8 : kThreads * 4;
            stage::arrive_expect_tx(mbar, total);
            int k = 3;
            for (int a = 1; a < arrays; ++a)
                for (int c = 0; c < planes[a]; ++c, ++k)
                    stage::copy(mlp::smem_addr(&sm.in.planes[k][0]), src[a] + c * pitch + start, bytes, mbar);
            const double* dsrc[4] = {in.temperature, in.water, cst.dry_mass, in.gas_moles};
            const float* fsrc[3] = {cst.volume, cst.gas_rate, in.porosity};
            for (int k = 0; k < 4; ++k)
                if (m & (1u << k)) stage::copy(mlp::smem_addr(&sm.in.d[k][0]), dsrc[k] + start, kThreads * 8, mbar);
            for (int k = 0; k < 3; ++k)
                if (m & (16u << k)) stage::copy(mlp::smem_addr(&sm.in.f[k][0]), fsrc[k] + start, kThreads * 4, mbar);
        }
        stencil_and_gather();
        const bool arrived = __syncthreads_and(mlp::mbar_wait(mbar, 0, stage::kWaitPolls)) != 0;
        if (!arrived) {
            // Leave this block's particles unprocessed and report it; wait (bounded) for the copies
            // still in flight into this block's shared memory before leaving.
            if (tid == 0 && P.status) atomicExch(P.status, 1);
            mlp::mbar_wait(mbar, 0, stage::kWaitPolls);
            return;
        }
    } else {
        stencil_and_gather();
    }
    // This particle's plane arrays: from the staged copies or from global memory.
    auto ld_v3 = [&](const float* src, int plane0) {
        if constexpr (kStaged) return V3{{sm.in.planes[plane0][tid], sm.in.planes[plane0 + 1][tid], sm.in.planes[plane0 + 2][tid]}};
        else return load_v3(src, i, pitch);
    };
    auto ld_m3 = [&](const float* src, int plane0) {
        if constexpr (kStaged) {
            M3 r;
#pragma unroll
            for (int c = 0; c < 9; ++c) r.m[c] = sm.in.planes[plane0 + c][tid];
            return r;
        } else {
            return load_m3(src, i, pitch);
        }
    };
    float mass = 0.f, q[3] = {0.f, 0.f, 0.f}, A[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (valid) {
        M3 F = ld_m3(in.F, 15);
        float J = det3(F);
        M3 tau;
        float T_mat = 0.f;
        float rho_ref = P.density;
        double sat = 0.0;
        if (P.transport) {
            double T_old = (staged_scalars & 1u) ? sm.in.d[0][tid] : in.temperature[i];
            double Tn = T_old + dTp;
            double Wn = ((staged_scalars & 2u) ? sm.in.d[1][tid] : in.water[i]) * (1.0 + ratio);
            double dry = (staged_scalars & 4u) ? sm.in.d[2][tid] : cst.dry_mass[i];
            float V0 = (staged_scalars & 16u) ? sm.in.f[0][tid] : cst.volume[i];
            out.temperature[i] = Tn;
            out.water[i] = Wn;
            mass = (float)(dry + Wn);
            rho_ref = (float)((dry + Wn) / (double)V0);
            sat = Wn / ((double)P.water_density * (double)V0 * (double)J);
            T_mat = (float)Tn;
            if (P.gas) {
                double N = (staged_scalars & 8u) ? sm.in.d[3][tid] : in.gas_moles[i];
                if (!P.settling) {
                    double Tm = 0.5 * (T_old + Tn);
                    double z = (Tm - (double)P.peak) / (double)P.width;
                    const float rate = (staged_scalars & 32u) ? sm.in.f[1][tid]
                                                              : cst.gas_rate[cst.gas_rate_per_particle ? i : 0];
                    N += (double)(P.dt * P.density) * (double)rate * exp(-(z * z));
                }
                out.gas_moles[i] = N;
            }
        } else {
            mass = cst.mass[i];
            if (P.material == 1) T_mat = in.material_temperature[i];
        }
        if (P.material == 1) {
            tau = ld_m3(in.tau, 24);
            if (P.gas) {
                float n = (staged_scalars & 64u) ? sm.in.f[2][tid] : in.porosity[i];
                if (n <= 0.0f || n >= 1.0f || !isfinite(n) || J <= 0.0f) {
                    set_flag(flags.ding, 0);
                } else {
                    float p = (float)gas_pressure(out.gas_moles[i], T_mat, J, n);
                    float iso = J * (P.ambient - p);
#pragma unroll
                    for (int e = 0; e < 9; ++e) tau.m[e] += (e % 4) == 0 ? iso : iso * 0.0f;
                    float bulk = p * (1.0f + (1.0f - P.ding.initial_porosity + n) / n);
                    float wave = sqrtf((P.elastic_modulus + bulk) * J / rho_ref);
                    if (!isfinite(p) || wave * P.dt / P.dx > P.cfl) set_flag(flags.ding, 2);
                }
            }
        } else {
            if (!isfinite(J) || J <= 0.0f) {
                set_flag(flags.simulation, 0);
#pragma unroll
                for (int e = 0; e < 9; ++e) tau.m[e] = 0.0f;
            } else {
                float lj = logf(J);
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        float ffT = F.m[3 * r] * F.m[3 * c] + F.m[3 * r + 1] * F.m[3 * c + 1] + F.m[3 * r + 2] * F.m[3 * c + 2];
                        float id = r == c ? 1.0f : 0.0f;
                        tau.m[3 * r + c] = P.ding.mu * (ffT - id) + P.ding.lam * lj * id;
                    }
            }
        }
        if (P.transport) {
            float iso = J * P.water_stress * ((float)sat - P.s0);
#pragma unroll
            for (int e = 0; e < 9; ++e) tau.m[e] -= (e % 4) == 0 ? iso : iso * 0.0f;
        }
        float scale = P.dt * ((staged_scalars & 16u) ? sm.in.f[0][tid] : cst.volume[i]) * 4.0f / (P.dx * P.dx);
        M3 Cm = ld_m3(in.C, 6);
        V3 vel = ld_v3(in.v, 3);
#pragma unroll
        for (int e = 0; e < 9; ++e) A[e] = mass * Cm.m[e] - scale * tau.m[e];
        // w (m v + A (o - l) dx) = w (q + A dx o) with q = m v - A l dx.
#pragma unroll
        for (int r = 0; r < 3; ++r)
            q[r] = mass * vel.v[r] - (A[3 * r] * st.l[0] + A[3 * r + 1] * st.l[1] + A[3 * r + 2] * st.l[2]) * P.dx;
#pragma unroll
        for (int e = 0; e < 9; ++e) A[e] *= P.dx;
    }
    if constexpr (kStaged) __syncthreads();  // every thread has read its planes: the records reuse them
    {
#pragma unroll
        for (int ox = 0; ox < 3; ++ox)
#pragma unroll
            for (int oy = 0; oy < 3; ++oy) {
                const float wxy = st.w[0][ox] * st.w[1][oy];
#pragma unroll
                for (int oz = 0; oz < 3; ++oz) sm.rec.w[9 * ox + 3 * oy + oz][tid] = valid ? wxy * st.w[2][oz] : 0.f;
            }
        sm.rec.val[tid][0] = make_float4(mass, q[0], q[1], q[2]);
        sm.rec.val[tid][1] = make_float4(A[0], A[1], A[2], A[3]);
        sm.rec.val[tid][2] = make_float4(A[4], A[5], A[6], A[7]);
        sm.rec.a8[tid] = A[8];
    }
    const BlockBox bb = block_box(g.bounds, valid, st.b);  // synchronises the block
    for (int t = tid; t < bb.count; t += kThreads) sm.tile[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    __syncthreads();
    long long key = valid ? pack_base(st.b) : -1;
    long long prev = __shfl_up_sync(kFull, key, 1);
    unsigned starts = __ballot_sync(kFull, valid && (lane == 0 || prev != key));
    const int warp_base = tid & ~31;
    int ox, oy, oz;
    node_offset(lane < 27 ? lane : 0, ox, oy, oz);
    const float fo[3] = {(float)ox, (float)oy, (float)oz};
    while (starts) {
        int s = __ffs(starts) - 1;
        starts &= starts - 1;
        int e = starts ? __ffs(starts) - 1 : 32;
        int b0 = __shfl_sync(kFull, st.b[0], s), b1 = __shfl_sync(kFull, st.b[1], s), b2 = __shfl_sync(kFull, st.b[2], s);
        if (lane < 27) {
            // Node j receives sum_k w_jk (m_k, q_k + A_k o_j): accumulate sum w m, sum w q, sum w A
            // (paired accumulators, one packed multiply-add per pair) and apply the node's offset
            // o_j once per run.
            float2 mq0 = {0.f, 0.f}, q12 = {0.f, 0.f}, A01 = {0.f, 0.f}, A23 = {0.f, 0.f};
            float2 A45 = {0.f, 0.f}, A67 = {0.f, 0.f};
            float A8 = 0.f;
            const float* wj = sm.rec.w[lane];
#pragma unroll 2
            for (int k = warp_base + s; k < warp_base + e; ++k) {
                const float w = wj[k];
                const float2 ww = make_float2(w, w);
                const float4 v0 = sm.rec.val[k][0], v1 = sm.rec.val[k][1], v2 = sm.rec.val[k][2];
                mq0 = ffma2(ww, make_float2(v0.x, v0.y), mq0);
                q12 = ffma2(ww, make_float2(v0.z, v0.w), q12);
                A01 = ffma2(ww, make_float2(v1.x, v1.y), A01);
                A23 = ffma2(ww, make_float2(v1.z, v1.w), A23);
                A45 = ffma2(ww, make_float2(v2.x, v2.y), A45);
                A67 = ffma2(ww, make_float2(v2.z, v2.w), A67);
                A8 = fmaf(w, sm.rec.a8[k], A8);
            }
            const float am = mq0.x;
            const float aq[3] = {mq0.y, q12.x, q12.y};
            const float aA[9] = {A01.x, A01.y, A23.x, A23.y, A45.x, A45.y, A67.x, A67.y, A8};
            float ap[3];
#pragma unroll
            for (int r = 0; r < 3; ++r)
                ap[r] = aq[r] + (aA[3 * r] * fo[0] + aA[3 * r + 1] * fo[1] + aA[3 * r + 2] * fo[2]);
            if (bb.tiled) {
                float* cell = reinterpret_cast<float*>(&sm.tile[tile_index(bb, b0 + ox, b1 + oy, b2 + oz)]);
                atomicAdd(cell + 0, ap[0]);
                atomicAdd(cell + 1, ap[1]);
                atomicAdd(cell + 2, ap[2]);
                atomicAdd(cell + 3, am);
            } else {
                atomicAdd(g.pm + node_index(b0 + ox, b1 + oy, b2 + oz, P.R), make_float4(ap[0], ap[1], ap[2], am));
            }
        }
    }
    __syncthreads();
    for (int t = tid; t < bb.count; t += kThreads) {
        float4 v = sm.tile[t];
        if (v.w == 0.0f && v.x == 0.0f && v.y == 0.0f && v.z == 0.0f) continue;
        atomicAdd(g.pm + tile_node(bb, t, P.R), v);
    }
}

template <bool kStaged, bool kLoaf = false>
__global__ void __launch_bounds__(kThreads, 4) k_p2g(Params P, BkState in, BkState out, BkConstants cst, GridPtrs g,
                                                 BkFlags flags, float* max_residuals) {
    pdl_enter();
    if constexpr (kLoaf) fix_loaf_mode(P);
    p2g_body<kStaged>(P, in, out, cst, g, flags, max_residuals, grid_slot());
}

// ------------------------------------------------------ fused G2P + return
// The largest positive value over the warp's active lanes into *addr (nonnegative floats order as
// their bit patterns): one atomic per warp instead of one per lane on the same address.
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float value) {
    const unsigned mask = __activemask();
    const int v = (int)__reduce_max_sync(mask, (unsigned)__float_as_int(value > 0.0f ? value : 0.0f));
    if (v > 0 && (int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(reinterpret_cast<int*>(addr), v);
}

// G2P of one particle (transfer.py:73-109): writes x', v', C', F' and returns F', C'. False (and the
// stencil flag) when the stencil leaves the grid.
// v = sum w v_i and C = 4/dx^2 sum w v_i (o_i - l) dx, accumulated as the moments
// S = sum w v_i and M_c = sum w v_i o_ic with the stencil offsets o_i in {0, 1, 2} known at compile
// time; C_rc = 4/dx (M_rc - l_c S_r).
__device__ __forceinline__ bool g2p_gather(const Params& P, const BkState& in, const BkState& out, const GridPtrs& g,
                                           const BkFlags& flags, int64_t i, M3& Fn, M3& Cn) {
    const int64_t pitch = P.pitch;
    V3 xi = load_v3(in.x, i, pitch);
    Stencil st = make_stencil(xi, P.origin, P.dx, P.R);
    if (!st.valid) { set_flag(flags.simulation, 1); return false; }
    float nv[3] = {0.f, 0.f, 0.f}, mo[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float4* vbase = g.v + node_index(st.b[0], st.b[1], st.b[2], P.R);
    const int64_t R = P.R;
#pragma unroll
    for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy) {
            const float wxy = st.w[0][ox] * st.w[1][oy];
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                float w = wxy * st.w[2][oz];
                float4 u = __ldg(vbase + (ox * R + oy) * R + oz);
                float wu[3] = {w * u.x, w * u.y, w * u.z};
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    nv[r] += wu[r];
                    if (ox) mo[3 * r + 0] += (float)ox * wu[r];
                    if (oy) mo[3 * r + 1] += (float)oy * wu[r];
                    if (oz) mo[3 * r + 2] += (float)oz * wu[r];
                }
            }
        }
    float nc[9];
    const float kdx = 4.0f / P.dx;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) nc[3 * r + c] = kdx * (mo[3 * r + c] - st.l[c] * nv[r]);
    M3 F = load_m3(in.F, i, pitch);
    M3 G;
#pragma unroll
    for (int e = 0; e < 9; ++e) {
        Cn.m[e] = nc[e];
        G.m[e] = P.dt * nc[e] + ((e % 4) == 0 ? 1.0f : 0.0f);
    }
    Fn = matmul(G, F);
    V3 vo{{nv[0], nv[1], nv[2]}}, xo{{xi.v[0] + P.dt * nv[0], xi.v[1] + P.dt * nv[1], xi.v[2] + P.dt * nv[2]}};
    store_v3(out.v, i, pitch, vo);
    store_m3(out.C, i, pitch, Cn);
    store_v3(out.x, i, pitch, xo);
    store_m3(out.F, i, pitch, Fn);
    return true;
}

__device__ __forceinline__ void ding_store(const Params& P, const BkState& out, const BkDiagnostics& diag, int64_t i,
                                           float T, const DingParticleOut& o) {
    const int64_t pitch = P.pitch;
    store_m3(out.Fe, i, pitch, o.Fe);
    store_m3(out.tau, i, pitch, o.tau);
    out.porosity[i] = o.porosity;
    out.gelled[i] = o.gelled;
    if (!P.transport) out.material_temperature[i] = T;
    if (diag.plastic_gradients) store_m3(diag.plastic_gradients, i, pitch, o.Fp);
    if (diag.return_residuals) diag.return_residuals[i] = o.residual;
    if (diag.porosity_residuals) diag.porosity_residuals[i] = o.porosity_residual;
    atomic_max_nonneg(diag.max_residuals, o.residual);
    atomic_max_nonneg(diag.max_residuals + 1, o.porosity_residual);
}

// ------------------------------------------------------ return-map surrogate
struct SurrogateDev {
    const unsigned char* blob;
    float in_mean[8], in_scale[8], in_low[8], in_high[8], out_scale[4];
    float* samples;
    int32_t* sample_count;
    int sample_capacity, sample_stride, sample_offset;
    float* judge_error;
    int judge_stride;
    int32_t* path_counts;
};

SurrogateDev surrogate_dev(const BkReturnSurrogate* r) {
    SurrogateDev d{};
    if (!r) return d;
    d.blob = static_cast<const unsigned char*>(r->packed);
    for (int k = 0; k < 8; ++k) {
        d.in_mean[k] = r->norm.in_mean[k];
        d.in_scale[k] = r->norm.in_scale[k] != 0.0f ? r->norm.in_scale[k] : 1.0f;
        d.in_low[k] = r->in_low[k];
        d.in_high[k] = r->in_high[k];
    }
    for (int k = 0; k < 4; ++k) d.out_scale[k] = r->norm.out_scale[k];
    d.samples = r->samples;
    d.sample_count = r->sample_count;
    d.sample_capacity = r->sample_capacity;
    d.sample_stride = r->sample_stride > 0 ? r->sample_stride : 1;
    d.sample_offset = r->sample_offset;
    d.judge_error = r->judge_error;
    d.judge_stride = r->judge_stride;
    d.path_counts = r->path_counts;
    return d;
}

// a[k] for a runtime k in {0, 1, 2} without dynamic register indexing (which would move `a` to
// local memory).
__device__ __forceinline__ float sel3(const float* a, int k) { return k == 0 ? a[0] : (k == 1 ? a[1] : a[2]); }

// Singular-value order (descending) the network sees, from the values or their logs.
__device__ __forceinline__ void order3(const float* s, int* perm) {
    int a = 0, b = 1, c = 2, t;
    if (s[a] < s[b]) { t = a; a = b; b = t; }
    if (s[b] < s[c]) { t = b; b = c; c = t; }
    if (s[a] < s[b]) { t = a; a = b; b = t; }
    perm[0] = a; perm[1] = b; perm[2] = c;
}

// The 7 raw network inputs of a particle: sorted log singular values of the trial elastic
// gradient, effective temperature, water saturation, gas content, plastic volume strain.
__device__ __forceinline__ void surrogate_features(const Params& P, const BkState& out, const BkConstants& cst,
                                                   int64_t i, const DingPrelude& d, float por, float J,
                                                   const int* perm, float* f) {
#pragma unroll
    for (int k = 0; k < 3; ++k) f[k] = sel3(d.e, perm[k]);
    f[3] = d.T_eff;
    f[4] = P.transport ? (float)(out.water[i] / ((double)P.water_density * (double)cst.volume[i] * (double)J)) : 0.0f;
    f[5] = P.gas ? (float)out.gas_moles[i] : 0.0f;
    f[6] = logf(1.0f - P.ding.initial_porosity + por);
}

// True when the exact return map leaves the particle elastic (no overstress solve): the cheap
// path for which the exact map runs unchanged.
__device__ __forceinline__ bool ding_elastic(const DingParamsDev& D, const DingPrelude& d, float por) {
    const float* st = d.e;
    float tr = st[0] + st[1] + st[2];
    float ts[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) ts[k] = 2.0f * D.mu * st[k] + D.lam * tr;
    float mean = (ts[0] + ts[1] + ts[2]) / 3.0f;
    float dev[3] = {ts[0] - mean, ts[1] - mean, ts[2] - mean};
    float ty2 = d.ty * d.ty;
    float q = 1.5f * (dev[0] * dev[0] + dev[1] * dev[1] + dev[2] * dev[2]) / ty2;
    float p = mean * mean / ty2;
    if (D.coupled_porosity) {
        // elastic trial porosity Vp - 1 + n0 with Vp = 1 - n0 + n, as in solve_porosity's early exit
        double trial = 1.0 - (double)D.initial_porosity + (double)por - 1.0 + (double)D.initial_porosity;
        if (trial > 0.0 && trial < 1.0) return (double)q + pressure_coefficient64(trial) * (double)p <= 1.0;
        return false;
    }
    return q + porosity_coefficient(por) * p <= 1.0f;
}

// Close the return from predicted log principal strains e (SVD order, before volume corrections):
// tau = U diag(2 mu dev(e) + K mean(e)) U^T, Fe = U exp(e) V^T; in gas mode the end-state porosity
// is the plastic volume change Vp exp(tr eps_trial - tr e) - 1 + n0. False when that porosity
// leaves (0, 1), in which case the caller runs the exact map.
__device__ bool ding_surrogate(const DingParamsDev& D, const DingPrelude& d, float por, const M3& F_tot,
                               const float* e, int32_t* flags, DingParticleOut& out, bool need_fp) {
    const float mu = D.mu, bulk = 2.0f * D.mu + 3.0f * D.lam;
    float ret_por = por;
    if (D.coupled_porosity) {
        double dv = (double)d.e[0] + (double)d.e[1] + (double)d.e[2] - ((double)e[0] + e[1] + e[2]);
        double rp = (1.0 - (double)D.initial_porosity + (double)por) * exp(dv) - 1.0 + (double)D.initial_porosity;
        if (!(rp > 0.0 && rp < 1.0)) return false;
        ret_por = (float)rp;
    }
    const float eb = (e[0] + e[1] + e[2]) / 3.0f;
    float cs[3], ex[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        cs[k] = 2.0f * mu * (e[k] - eb) + bulk * eb;
        ex[k] = expf(e[k]);
    }
    const float* U = d.U.m;
    const float* V = d.V.m;
    M3 Fe, tau;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            Fe.m[3 * r + c] = (U[3 * r] * ex[0]) * V[3 * c] + (U[3 * r + 1] * ex[1]) * V[3 * c + 1] +
                              (U[3 * r + 2] * ex[2]) * V[3 * c + 2];
            tau.m[3 * r + c] = (U[3 * r] * cs[0]) * U[3 * c] + (U[3 * r + 1] * cs[1]) * U[3 * c + 1] +
                               (U[3 * r + 2] * cs[2]) * U[3 * c + 2];
        }
    if (!D.coupled_porosity && porosity_coefficient(por) == 0.0f) {
        float scale = cbrtf(d.det_trial / det3(Fe));
#pragma unroll
        for (int k = 0; k < 9; ++k) Fe.m[k] *= scale;
    }
    ding_close(D, por, FInRegs{F_tot}, ret_por, Fe, flags, out, need_fp);
    out.tau = tau;
    out.residual = 0.0f;
    out.porosity_residual = 0.0f;
    out.yield_stress = d.ty;
    out.viscosity = d.eta;
    out.gelled = d.gel;
#pragma unroll
    for (int k = 0; k < 3; ++k) out.e[k] = e[k];
    out.yielded = true;
    return true;
}

// 8 blocks of 128 threads per SM (64 registers): the return map's dependent float64 chains are
// latency bound, so resident warps outweigh the spilled registers (measured at 3 to 12 blocks per
// SM: 8 is fastest for both elastic and yielding particles). With `sg.samples` set (harvest),
// yielding particles on the sampling stride append (features, return) rows.
__device__ __forceinline__ void g2p_return_particle(const Params& P, const BkState& in, const BkState& out,
                                                    const BkConstants& cst, const GridPtrs& g, const BkDiagnostics& diag,
                                                    const BkFlags& flags, const SurrogateDev& sg, int64_t i) {
    M3 Fn, Cn;
    if (!g2p_gather(P, in, out, g, flags, i, Fn, Cn)) return;
    if (P.material != 1) return;
    const int64_t pitch = P.pitch;
    float T = P.transport ? (float)out.temperature[i] : in.material_temperature[i];
    const float por = in.porosity[i];
    DingPrelude d;
    if (!ding_prelude(P.ding, load_m3(in.Fe, i, pitch), por, in.gelled[i], Cn, T, __ldg(cst.viscosity_parameter),
                      flags.ding, d))
        return;
    DingParticleOut o;
    ding_exact(P.ding, d, por, FStored{out.F, i, pitch}, flags.ding, o, diag.plastic_gradients != nullptr);
    ding_store(P, out, diag, i, T, o);
    if (sg.samples && o.yielded && i % sg.sample_stride == sg.sample_offset) {
        int slot = atomicAdd(sg.sample_count, 1);
        if (slot < sg.sample_capacity) {
            int perm[3];
            order3(d.e, perm);
            float f[7];
            surrogate_features(P, out, cst, i, d, por, det3(FStored{out.F, i, pitch}.get()), perm, f);
            float* row = sg.samples + (int64_t)slot * 12;
#pragma unroll
            for (int k = 0; k < 7; ++k) row[k] = f[k];
#pragma unroll
            for (int k = 0; k < 3; ++k) row[7 + k] = sel3(o.e, perm[k]) - f[k];
            row[10] = 0.0f;
            row[11] = 0.0f;
        }
    }
}

// Shared-memory node tile of the transport prescatter in k_g2p_return (128 particles per block).
constexpr int kG2PTile = 256;
using G2PTransportTile = TransportTile<128, kG2PTile, 4, false>;

template <bool kRef = false>
__device__ __forceinline__ void g2p_return_body(Arg<Params, kRef> P, Arg<BkState, kRef> in,
                                                Arg<BkState, kRef> out, Arg<BkConstants, kRef> cst, Arg<GridPtrs, kRef> g,
                                                Arg<BkDiagnostics, kRef> diag, Arg<BkFlags, kRef> flags, Arg<SurrogateDev, kRef> sg,
                                                Slot sl) {
    extern __shared__ __align__(16) unsigned char g2p_smem[];
    const int64_t i = sl.block * (int64_t)blockDim.x + threadIdx.x;
    if (sl.block == 0 && threadIdx.x < 6) {
        // This substep's box becomes the box the next substep clears; the active box restarts empty.
        g.bounds[6 + threadIdx.x] = g.bounds[threadIdx.x];
        g.bounds[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
    }
    if (i < P.n) g2p_return_particle(P, in, out, cst, g, diag, flags, sg, i);
    if (P.prescatter_next) {
        // The next substep's scalar P2G (thermal_water.py:108-137) from the state just written:
        // x' and F' by this thread (read back with plain loads), T' and W' by this substep's P2G.
        // The grid update has zeroed the transport fields over this substep's box and restarted
        // the prescatter box bounds[12..17]. Uniform branch: every thread of the block scatters.
        G2PTransportTile& sm = *reinterpret_cast<G2PTransportTile*>(g2p_smem);
        const int64_t pitch = P.pitch;
        bool valid = false;
        Stencil st;
        st.b[0] = st.b[1] = st.b[2] = 0;
        double val[4] = {0.0, 0.0, 0.0, 0.0};
        if (i < P.n) {
            const float* xs = out.x;
            const V3 x{{xs[i], xs[pitch + i], xs[2 * pitch + i]}};
            st = make_stencil(x, P.origin, P.dx, P.R);
            valid = st.valid;
            if (valid) {
                const double cap = cst.capacity[i];
                val[0] = (double)cst.volume[i] * (double)det3(FStored{out.F, i, pitch}.get());
                val[1] = cap;
                val[2] = cap * out.temperature[i];
                val[3] = out.water[i];
            }
        }
        transport_scatter_block<128, kG2PTile, 4, 0, false>(sm, P, g, g.bounds + 12, valid, st, val);
    }
}

// kLoaf instances also fix whether the next substep's transport fields are scattered (kPrescatter).
template <bool kLoaf = false, bool kPrescatter = false>
__global__ void __launch_bounds__(128, 8) k_g2p_return(Params P, BkState in, BkState out, BkConstants cst, GridPtrs g,
                                                   BkDiagnostics diag, BkFlags flags, SurrogateDev sg) {
    pdl_enter();
    if constexpr (kLoaf) {
        fix_loaf_mode(P);
        P.prescatter_next = kPrescatter;
        diag.plastic_gradients = diag.return_residuals = diag.porosity_residuals = nullptr;
        sg.samples = nullptr;
    }
    g2p_return_body(P, in, out, cst, g, diag, flags, sg, grid_slot());
}

// G2P + return map with the learned surrogate: a persistent CTA walks 128-particle tiles and
// evaluates the network for each on the tensor cores (bk_mlp.cuh), so the weights are staged,
// the tensor memory allocated and the mbarrier initialised once per CTA. Yielding particles inside
// the training range take the surrogate's return; all others (elastic, out of range, invalid
// porosity) the exact map. The trial gradient's SVD stops at float32 convergence (svd3f<false>):
// its float64 finishing sweep only matters at the reference's rounding level, far below the
// network's error.
template <bool kRef = false>
__device__ __forceinline__ void g2p_return_surrogate_body(Arg<Params, kRef> P, Arg<BkState, kRef> in, Arg<BkState, kRef> out,
                                                          Arg<BkConstants, kRef> cst, Arg<GridPtrs, kRef> g,
                                                          Arg<BkDiagnostics, kRef> diag, Arg<BkFlags, kRef> flags,
                                                          Arg<SurrogateDev, kRef> sg, Slot sl) {
    __shared__ mlp::TileSmem ts;
    __shared__ int s_counts[3];
    mlp::tile_setup(ts, sg.blob);
    if (threadIdx.x < 3) s_counts[threadIdx.x] = 0;
    if (sl.block == 0 && threadIdx.x < 6) {
        g.bounds[6 + threadIdx.x] = g.bounds[threadIdx.x];
        g.bounds[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
    }
    __syncthreads();
    const int64_t pitch = P.pitch;
    uint32_t phase = 0;
    for (int64_t base = (int64_t)sl.block * 128; base < P.n; base += (int64_t)sl.blocks * 128) {
        const int64_t i = base + threadIdx.x;
        M3 Fn, Cn;
        bool ding = false, use_mlp = false;
        DingPrelude d;
        float T = 0.f, por = 0.f, x[7] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int perm[3] = {0, 1, 2};
        if (i < P.n && g2p_gather(P, in, out, g, flags, i, Fn, Cn) && P.material == 1) {
            T = P.transport ? (float)out.temperature[i] : in.material_temperature[i];
            por = in.porosity[i];
            ding = ding_prelude<false>(P.ding, load_m3(in.Fe, i, pitch), por, in.gelled[i], Cn, T,
                                __ldg(cst.viscosity_parameter), flags.ding, d);
            if (ding && !ding_elastic(P.ding, d, por)) {
                order3(d.e, perm);
                float f[7];
                surrogate_features(P, out, cst, i, d, por, det3(Fn), perm, f);
                use_mlp = true;
#pragma unroll
                for (int k = 0; k < 7; ++k) {
                    use_mlp = use_mlp && f[k] >= sg.in_low[k] && f[k] <= sg.in_high[k];
                    x[k] = (f[k] - sg.in_mean[k]) / sg.in_scale[k];
                }
            }
        }
        float y[3] = {0.f, 0.f, 0.f};
        // A tile whose particles all take the exact map (elastic, or outside the training range)
        // skips the network; the barrier makes the decision uniform across the CTA.
        const bool any_mlp = __syncthreads_or(use_mlp) != 0;
        const bool tile_ok = any_mlp ? mlp::tile_eval(ts, x, use_mlp, y, phase) : true;
        int path = -1;
        if (ding) {
            DingParticleOut o;
            bool done = false;
            if (use_mlp && tile_ok) {
                // y is in the sorted order: singular value j has rank r_j with perm[r_j] = j.
                float e[3];
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const int r = perm[0] == j ? 0 : (perm[1] == j ? 1 : 2);
                    e[j] = d.e[j] + sel3(y, r) * sel3(sg.out_scale, r);
                }
                done = ding_surrogate(P.ding, d, por, Fn, e, flags.ding, o, diag.plastic_gradients != nullptr);
                // Judged in whole warps, so that the exact map's cost falls on 1 warp in judge_stride.
                if (done && sg.judge_error && sg.judge_stride > 0 && (i >> 5) % sg.judge_stride == 0) {
                    DingParticleOut ex;
                    ding_exact(P.ding, d, por, FInRegs{Fn}, nullptr, ex, false);  // judge only: no flags
                    float err = 0.f;
#pragma unroll
                    for (int k = 0; k < 3; ++k) err = fmaxf(err, fabsf(ex.e[k] - e[k]));
                    atomic_max_nonneg(sg.judge_error, err);
                }
            }
            if (!done) ding_exact(P.ding, d, por, FInRegs{Fn}, flags.ding, o, diag.plastic_gradients != nullptr);
            path = done ? 1 : (o.yielded ? 2 : 0);
            ding_store(P, out, diag, i, T, o);
        }
        if (sg.path_counts && path >= 0) atomicAdd(&s_counts[path], 1);
        __syncthreads();
        if (ts.failed) {  // read after a barrier, so every thread takes the same branch
            if (threadIdx.x == 0 && P.status) atomicExch(P.status, 1);  // later tiles stay unprocessed
            break;
        }
    }
    mlp::tile_teardown(ts);
    if (sg.path_counts && threadIdx.x < 3 && s_counts[threadIdx.x]) atomicAdd(sg.path_counts + threadIdx.x, s_counts[threadIdx.x]);
}

template <bool kLoaf = false>
__global__ void __launch_bounds__(128, 4) k_g2p_return_surrogate(Params P, BkState in, BkState out, BkConstants cst,
                                                             GridPtrs g, BkDiagnostics diag, BkFlags flags,
                                                             SurrogateDev sg) {
    pdl_enter();
    if constexpr (kLoaf) {
        fix_loaf_mode(P);
        diag.plastic_gradients = diag.return_residuals = diag.porosity_residuals = nullptr;
        sg.samples = nullptr;
    }
    g2p_return_surrogate_body(P, in, out, cst, g, diag, flags, sg, grid_slot());
}

// ------------------------------------------------------------ materialize
__global__ void k_materialize(Params P, BkState s, BkConstants cst, float* Fp, float* T_mat, float* rho,
                              float* yield, float* visc, double* gas_p, double* sat, float* mass) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const int64_t pitch = P.pitch;
    M3 F = load_m3(s.F, i, pitch);
    float J = det3(F);
    float T = 0.f;
    if (P.transport) {
        double W = s.water[i], dry = cst.dry_mass[i];
        double V0 = (double)cst.volume[i];
        T = (float)s.temperature[i];
        if (rho) rho[i] = (float)((dry + W) / V0);
        if (sat) sat[i] = W / ((double)P.water_density * V0 * (double)J);
        if (mass) mass[i] = (float)(dry + W);
    } else if (P.material == 1) {
        T = s.material_temperature[i];
        if (rho) rho[i] = P.density;
    }
    if (P.material != 1) return;
    if (T_mat) T_mat[i] = T;
    if (Fp) store_m3(Fp, i, pitch, matmul(inverse3(load_m3(s.Fe, i, pitch)), F));
    const DingParamsDev& D = P.ding;
    float ty = D.yield_stress, eta = __ldg(cst.viscosity_parameter);
    if (D.temperature_enabled) {
        float Teff = s.gelled[i] ? D.knots[3] : T;
        ty = D.yield_stress * temperature_factor(Teff, D.knots, D.yield_factors);
        eta = eta * temperature_factor(Teff, D.knots, D.viscosity_factors);
    }
    if (yield) yield[i] = ty;
    if (visc) visc[i] = eta;
    if (gas_p && P.gas) {
        float n = s.porosity[i];
        if (n > 0.0f && n < 1.0f) gas_p[i] = gas_pressure(s.gas_moles[i], T, J, n);
    }
}

// physics/thermal_water.py:225-226 for the face-owning particles (the only ones whose loss or
// exchange changes): accumulators += dt * per-owner rate.
__global__ void k_surface_accumulate(int64_t owners_n, const int32_t* __restrict__ owners,
                                     const double* __restrict__ heat, const double* __restrict__ loss, double dt,
                                     double* __restrict__ water_losses, double* __restrict__ heat_exchanges) {
    int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (o >= owners_n) return;
    int p = owners[o];
    water_losses[p] += dt * loss[o];
    heat_exchanges[p] += dt * heat[o];
}

unsigned blocks_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

#define BK_REQUIRE(cond, msg) do { if (!(cond)) return fail(BK_ERR_ARGUMENT, msg); } while (0)

// The argument checks of bk_substep (also applied to every instance of a batch).
int check_substep_args(const BkSubstepParams* params, const BkState* in, const BkState* out,
                       const BkConstants* constants, const BkGrid* grid, const BkSurface* surface,
                       const BkDiagnostics* diagnostics, const BkFlags* flags, int32_t phases) {
    BK_REQUIRE(params && in && out && constants && grid && diagnostics && flags, "bk_substep: null argument");
    const BkSubstepParams& p = *params;
    BK_REQUIRE(p.n >= 0 && p.pitch >= p.n, "bk_substep: bad particle count/pitch");
    BK_REQUIRE(p.resolution >= 4 && p.resolution < (1 << 20) && p.spacing > 0.0f, "bk_substep: bad grid");
    BK_REQUIRE(grid->node_pm && grid->node_v && grid->bounds, "bk_substep: missing grid arrays");
    BK_REQUIRE((((uintptr_t)grid->node_pm | (uintptr_t)grid->node_v) & 15) == 0, "bk_substep: grid not 16-byte aligned");
    BK_REQUIRE(in->x && in->v && in->C && in->F && out->x && out->v && out->C && out->F, "bk_substep: missing state");
    BK_REQUIRE(flags->simulation && flags->ding && flags->transport && diagnostics->max_residuals,
               "bk_substep: missing flags");
    if (p.material == 1)
        BK_REQUIRE(in->Fe && in->tau && in->porosity && in->gelled && out->Fe && out->tau && out->porosity &&
                   out->gelled && constants->viscosity_parameter, "bk_substep: missing Ding state");
    if (p.material == 1 && !p.transport)
        BK_REQUIRE(in->material_temperature && out->material_temperature, "bk_substep: missing Ding temperature");
    if (p.transport) {
        BK_REQUIRE(surface && in->temperature && in->water && out->temperature && out->water && constants->capacity &&
                   constants->dry_mass && constants->heat_parameter && grid->node_dT_ratio,
                   "bk_substep: missing transport arrays");
        for (int k = 0; k < 7; ++k) BK_REQUIRE(grid->fields[k] != nullptr, "bk_substep: missing node field");
        BK_REQUIRE(((uintptr_t)grid->node_dT_ratio & 15) == 0, "bk_substep: node_dT_ratio not 16-byte aligned");
    } else {
        BK_REQUIRE(constants->mass != nullptr, "bk_substep: missing particle masses");
    }
    if (p.gas)
        BK_REQUIRE(p.transport && p.material == 1 && in->gas_moles && out->gas_moles && constants->gas_rate,
                   "bk_substep: gas mode needs transport, the Ding model and gas arrays");
    if (p.transport_prescattered || p.transport_prescatter_next || p.transport_prescatter_stale)
        BK_REQUIRE(p.transport && !p.keep_transport_fields,
                   "bk_substep: the transport prescatter needs transport and a grid update that clears the fields");
    if (p.transport_prescatter_next)
        BK_REQUIRE(!(p.surrogate && p.surrogate->packed) && (phases & BK_PHASE_MECHANICS),
                   "bk_substep: the transport prescatter runs in the exact G2P kernel of a mechanics phase");
    return BK_OK;
}

}  // namespace

extern "C" {

int bk_substep(const BkSubstepParams* params, const BkState* in, BkState* out, const BkConstants* constants,
               BkGrid* grid, BkSurface* surface, BkDiagnostics* diagnostics, BkFlags* flags, int32_t phases,
               void* stream) {
    if (int rc = check_substep_args(params, in, out, constants, grid, surface, diagnostics, flags, phases)) return rc;
    const BkSubstepParams& p = *params;
    if (p.n == 0) return BK_OK;
    Params P = to_params(p);
    GridPtrs g = grid_ptrs(*grid);
    cudaStream_t s = S(stream);
    const unsigned particle_blocks = blocks_for(p.n, kThreads);
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const unsigned box_blocks = (unsigned)sms * 4;
    cudaError_t e = cudaSuccess;
    if ((phases & BK_PHASE_TRANSPORT) && p.transport) {
        if (surface->vertex_count > 0) {
            {
                int rec = profile_begin("surface_vertices", s);
                const unsigned nv = (unsigned)surface->vertex_count;
                switch (vertex_block_threads(surface->vertex_count, surface->binding_count)) {
                    case 256: e = launch_chained(k_surface_vertices<256>, nv, 256, 0, s, P, in->x, in->F, *surface); break;
                    case 128: e = launch_chained(k_surface_vertices<128>, nv, 128, 0, s, P, in->x, in->F, *surface); break;
                    default:
                        e = launch_chained(k_surface_vertices<32>, vertex_launch_blocks(nv, 32), vertex_launch_threads(32),
                                           0, s, P, in->x, in->F, *surface);
                        break;
                }
                profile_end(rec, s);
            }
            if (int rc = check_chained(e, "bk_substep/surface_vertices")) return rc;
        }
        if (surface->owner_count > 0) {
            {
                int rec = profile_begin("surface_owners", s);
                e = launch_chained(k_surface_owners, owner_blocks(surface->owner_count, p.n), kOwnerThreads, 0, s, P,
                                   *in, *constants, *surface, g, flags->simulation,
                                   (int)owners_tiled(surface->owner_count, p.n));
                profile_end(rec, s);
            }
            if (int rc = check_chained(e, "bk_substep/surface_owners")) return rc;
        }
        if (!p.transport_prescattered) {
            if (p.transport_prescatter_stale) {
                e = launch_chained(k_clear_prescatter, box_blocks, kThreads, 0, s, P, g);
                if (int rc = check_chained(e, "bk_substep/clear_prescatter")) return rc;
            }
            {
                int rec = profile_begin("transport_scatter", s);
                e = launch_chained(k_transport_scatter, particle_blocks, kThreads, 0, s, P, *in, *constants, g,
                                   flags->simulation);
                profile_end(rec, s);
            }
            if (int rc = check_chained(e, "bk_substep/transport_scatter")) return rc;
        }
        {
            int rec = profile_begin("diffuse", s);
            e = launch_chained(k_diffuse, box_blocks, kDiffThreads, 0, s, P, g, flags->transport);
            profile_end(rec, s);
        }
        if (int rc = check_chained(e, "bk_substep/diffuse")) return rc;
    }
    if (phases & BK_PHASE_MECHANICS) {
        {
            int rec = profile_begin("clear_previous", s);
            e = launch_chained(k_clear_previous, box_blocks, kThreads, 0, s, P, g);
            profile_end(rec, s);
        }
        if (int rc = check_chained(e, "bk_substep/clear_previous")) return rc;
        {
            int rec = profile_begin("p2g", s);
            // Bulk staging needs 16-byte aligned plane starts: a pitch that is a multiple of 4 floats
            // and 16-byte aligned array bases.
            const bool staged = p.pitch % 4 == 0 && (p2g_stage_bases(p, *in, *constants) & 15) == 0;
            if (int rc = allow_smem(staged ? (loaf_mode(p, *diagnostics) ? (const void*)k_p2g<true, true> : (const void*)k_p2g<true>)
                                           : (loaf_mode(p, *diagnostics) ? (const void*)k_p2g<false, true> : (const void*)k_p2g<false>),
                                    kP2GSmemBytes, "bk_substep/p2g"))
                return rc;
            const bool loaf = loaf_mode(p, *diagnostics);
            auto* kernel = staged ? (loaf ? k_p2g<true, true> : k_p2g<true>) : (loaf ? k_p2g<false, true> : k_p2g<false>);
            e = launch_chained(kernel, particle_blocks, kThreads, kP2GSmemBytes, s, P, *in, *out, *constants, g, *flags,
                               diagnostics->max_residuals);
            profile_end(rec, s);
        }
        if (int rc = check_chained(e, "bk_substep/p2g")) return rc;
        {
            int rec = profile_begin("grid_update", s);
            e = launch_chained(k_grid_update, box_blocks, kThreads, 0, s, P, g);
            profile_end(rec, s);
        }
        if (int rc = check_chained(e, "bk_substep/grid_update")) return rc;
        const SurrogateDev sg = surrogate_dev(p.surrogate);
        if (sg.blob && p.material == 1) {
            int rec = profile_begin("g2p_return_surrogate", s);
            const unsigned tiles = blocks_for(p.n, 128);
            const unsigned persistent = (unsigned)sms * 4;
            e = launch_chained(loaf_mode(p, *diagnostics) ? k_g2p_return_surrogate<true> : k_g2p_return_surrogate<false>,
                               tiles < persistent ? tiles : persistent, 128, 0, s, P, *in, *out, *constants, g,
                               *diagnostics, *flags, sg);
            profile_end(rec, s);
        } else {
            int rec = profile_begin("g2p_return", s);
            const size_t smem = p.transport_prescatter_next ? sizeof(G2PTransportTile) : 0;
            auto* kernel = !loaf_mode(p, *diagnostics)       ? k_g2p_return<false>
                           : p.transport_prescatter_next ? k_g2p_return<true, true>
                                                         : k_g2p_return<true, false>;
            e = launch_chained(kernel, blocks_for(p.n, 128), 128, smem, s, P, *in, *out, *constants, g, *diagnostics,
                               *flags, sg);
            profile_end(rec, s);
        }
        if (int rc = check_chained(e, "bk_substep/g2p_return")) return rc;
    }
    return BK_OK;
}

int bk_surface_accumulate(const BkSurface* surface, float time_step, double* water_losses, double* heat_exchanges,
                          void* stream) {
    BK_REQUIRE(surface && water_losses && heat_exchanges, "bk_surface_accumulate: null argument");
    if (surface->owner_count == 0) return BK_OK;
    BK_REQUIRE(surface->owners && surface->owner_heat && surface->owner_loss, "bk_surface_accumulate: missing owners");
    k_surface_accumulate<<<blocks_for(surface->owner_count, kThreads), kThreads, 0, S(stream)>>>(
        surface->owner_count, surface->owners, surface->owner_heat, surface->owner_loss, (double)time_step,
        water_losses, heat_exchanges);
    return check_launch("bk_surface_accumulate");
}

int bk_materialize(const BkSubstepParams* params, const BkState* state, const BkConstants* constants,
                   float* plastic_gradients, float* material_temperature, float* reference_density,
                   float* yield_stress, float* viscosity, double* gas_pressure, double* saturation,
                   float* particle_mass, void* stream) {
    BK_REQUIRE(params && state && constants, "bk_materialize: null argument");
    const BkSubstepParams& p = *params;
    BK_REQUIRE(p.n >= 0 && p.pitch >= p.n, "bk_materialize: bad particle count/pitch");
    if (p.n == 0) return BK_OK;
    BK_REQUIRE(state->F != nullptr, "bk_materialize: missing F");
    if (p.transport)
        BK_REQUIRE(state->temperature && state->water && constants->dry_mass && constants->volume,
                   "bk_materialize: missing transport arrays");
    if (p.material == 1)
        BK_REQUIRE(state->Fe && state->gelled && state->porosity && constants->viscosity_parameter &&
                   (p.transport || state->material_temperature), "bk_materialize: missing Ding arrays");
    if (p.gas && gas_pressure) BK_REQUIRE(state->gas_moles != nullptr, "bk_materialize: missing gas moles");
    k_materialize<<<blocks_for(p.n, kThreads), kThreads, 0, S(stream)>>>(
        to_params(p), *state, *constants, plastic_gradients, material_temperature, reference_density, yield_stress,
        viscosity, gas_pressure, saturation, particle_mass);
    return check_launch("bk_materialize");
}

}  // extern "C"

// ===================================================================== batched substeps
// Many independent simulators advanced by one launch per stage: each block of a batched launch
// finds its instance in a device table (a binary search over the stage's first-block prefix),
// copies that instance's entry into shared memory and runs the same kernel body as a plain
// launch, with its index among the instance's blocks. The blocks an instance gets per stage are
// the ones its own launch would use (particles, vertices, owners), or for the node-box passes a
// share that grows with its particle count, so a batch of small bodies fills the GPU.
namespace {

enum BatchStage { kStVertices, kStOwners, kStScatter, kStDiffuse, kStClear, kStP2G, kStGrid, kStG2P, kStSurrogate,
                  kBatchStages };

struct BatchEntry {
    Params P;
    BkState in, out;
    BkConstants cst;
    GridPtrs g;
    BkSurface sf;
    BkDiagnostics diag;
    BkFlags flags;
    SurrogateDev sg;   // sf carries the surface accumulators of `out`
    int prescatter_ok;  // takes part in the transport prescatter
    int owners_tiled;   // the surface terms take the tiled form (owners_tiled)
};
static_assert(sizeof(BatchEntry) % 4 == 0, "entries are copied as 4-byte words");

struct BatchArgs {
    const BatchEntry* entries;  // [2][count]: parity 0 steps states[0] -> states[1], parity 1 back
    const uint32_t* first;      // [kBatchStages][count + 1]: first block of each instance per stage
    const int32_t* owner;       // the instance of every block of every stage, stage by stage
    uint32_t owner_offset[kBatchStages];  // where each stage's blocks start in `owner`
    int count, parity, prescattered, prescatter_next;
};

// The instance that owns this block in `stage` (one load from the block map) and the block's slot
// within it.
__device__ __forceinline__ Slot batch_find(const BatchArgs& b, int stage, int& k) {
    k = __ldg(b.owner + b.owner_offset[stage] + blockIdx.x);
    const uint32_t* f = b.first + (size_t)stage * (b.count + 1);
    const uint32_t f0 = __ldg(f + k), f1 = __ldg(f + k + 1);
    return Slot{(int)(blockIdx.x - f0), (int)(f1 - f0)};
}

// Copies the block's entry into shared memory with this call's prescatter flags. Every thread of
// the block calls it (it synchronises the block).
__device__ __forceinline__ Slot batch_load(const BatchArgs& b, int stage, BatchEntry& e) {
    int k;
    const Slot sl = batch_find(b, stage, k);
    const int* src = reinterpret_cast<const int*>(b.entries + (size_t)b.parity * b.count + k);
    int* dst = reinterpret_cast<int*>(&e);
    for (int w = threadIdx.x; w < (int)(sizeof(BatchEntry) / 4); w += blockDim.x) dst[w] = __ldg(src + w);
    __syncthreads();
    if (threadIdx.x == 0) {
        e.P.prescattered = b.prescattered && e.prescatter_ok;
        e.P.prescatter_next = b.prescatter_next && e.prescatter_ok;
        e.P.prescatter_stale = 0;
    }
    __syncthreads();
    return sl;
}

template <int kBlock>
__global__ void __launch_bounds__(kBlock == 32 ? 32 * kVertexWarps : kBlock) kb_surface_vertices(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStVertices, e);
    surface_vertices_body<kBlock, true>(e.P, e.in.x, e.in.F, e.sf, sl);
}

__global__ void __launch_bounds__(kOwnerThreads) kb_surface_owners(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStOwners, e);
    surface_owners_body<true>(e.P, e.in, e.cst, e.sf, e.g, e.flags.simulation, e.owners_tiled != 0, sl);
}

__global__ void __launch_bounds__(kThreads) kb_transport_scatter(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStScatter, e);
    if (e.P.prescattered) return;  // fields scattered ahead by this instance's previous G2P
    transport_scatter_body<true>(e.P, e.in, e.cst, e.g, e.flags.simulation, sl);
}

__global__ void __launch_bounds__(kDiffThreads) kb_diffuse(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStDiffuse, e);
    diffuse_body<true>(e.P, e.g, e.flags.transport, sl);
}

__global__ void __launch_bounds__(kThreads) kb_clear_previous(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStClear, e);
    clear_previous_body<true>(e.P, e.g, sl);
}

template <bool kStaged>
__global__ void __launch_bounds__(kThreads, 4) kb_p2g(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStP2G, e);
    p2g_body<kStaged, true>(e.P, e.in, e.out, e.cst, e.g, e.flags, e.diag.max_residuals, sl);
}

__global__ void __launch_bounds__(kThreads) kb_grid_update(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStGrid, e);
    grid_update_body<true>(e.P, e.g, sl);
}

__global__ void __launch_bounds__(128, 8) kb_g2p_return(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStG2P, e);
    g2p_return_body<true>(e.P, e.in, e.out, e.cst, e.g, e.diag, e.flags, e.sg, sl);
}

__global__ void __launch_bounds__(128, 4) kb_g2p_return_surrogate(BatchArgs b) {
    __shared__ BatchEntry e;
    const Slot sl = batch_load(b, kStSurrogate, e);
    g2p_return_surrogate_body<true>(e.P, e.in, e.out, e.cst, e.g, e.diag, e.flags, e.sg, sl);
}

}  // namespace

struct BkBatch {
    int count = 0;
    BatchEntry* entries = nullptr;  // device [2][count]
    uint32_t* first = nullptr;      // device [kBatchStages][count + 1]
    int32_t* owner = nullptr;       // device: instance of each block, stage by stage
    uint32_t owner_offset[kBatchStages] = {};
    uint32_t total[kBatchStages] = {};
    int vertex_block = 32;
    bool staged = true;             // every instance allows the bulk-staged P2G
    bool all_prescatter = true;     // every transport instance takes part in the prescatter
    bool any_transport = false;
};

extern "C" {

int bk_batch_create(const BkBatchInstance* instances, int32_t count, BkBatch** batch) {
    BK_REQUIRE(instances && batch && count > 0, "bk_batch_create: null argument or empty batch");
    *batch = nullptr;
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    std::vector<BatchEntry> entries(2 * (size_t)count);
    std::vector<uint32_t> first((size_t)kBatchStages * (count + 1), 0);
    int64_t particles = 0, vertices = 0, bindings = 0;
    for (int k = 0; k < count; ++k) {
        particles += instances[k].params.n;
        if (instances[k].params.transport && instances[k].params.n > 0) {
            vertices += instances[k].surface.vertex_count;
            bindings += instances[k].surface.binding_count;
        }
    }
    BkBatch host;
    host.count = count;
    host.vertex_block = vertex_block_threads(vertices, bindings);  // one block size for the whole launch
    for (int k = 0; k < count; ++k) {
        const BkBatchInstance& in = instances[k];
        const BkSubstepParams& p = in.params;
        const bool surrogate = p.surrogate && p.surrogate->packed && p.material == 1;
        for (int parity = 0; parity < 2; ++parity) {
            const BkState& a = in.states[parity];
            const BkState& b = in.states[1 - parity];
            BkSubstepParams q = p;
            q.transport_prescattered = q.transport_prescatter_next = q.transport_prescatter_stale = 0;
            if (int rc = check_substep_args(&q, &a, &b, &in.constants, &in.grid, &in.surface, &in.diagnostics,
                                            &in.flags, BK_PHASE_TRANSPORT | BK_PHASE_MECHANICS))
                return rc;
            if (p.transport)
                BK_REQUIRE(in.water_losses[1 - parity] && in.heat_exchanges[1 - parity],
                           "bk_batch_create: missing surface accumulators");
            BatchEntry& e = entries[(size_t)parity * count + k];
            e.P = to_params(q);
            e.in = a;
            e.out = b;
            e.cst = in.constants;
            e.g = grid_ptrs(in.grid);
            e.sf = in.surface;
            e.sf.accumulate_water_losses = p.transport ? in.water_losses[1 - parity] : nullptr;
            e.sf.accumulate_heat_exchanges = p.transport ? in.heat_exchanges[1 - parity] : nullptr;
            e.sf.accumulate_time_step = p.time_step;
            e.diag = in.diagnostics;
            e.flags = in.flags;
            e.sg = surrogate_dev(surrogate ? p.surrogate : nullptr);
            e.prescatter_ok = p.transport && !p.keep_transport_fields && !surrogate;
            e.owners_tiled = owners_tiled(in.surface.owner_count, p.n);
            host.staged = host.staged && p.pitch % 4 == 0 && (p2g_stage_bases(p, a, in.constants) & 15) == 0;
        }
        host.any_transport = host.any_transport || p.transport;
        if (p.transport && (p.keep_transport_fields || surrogate)) host.all_prescatter = false;
        uint32_t blocks[kBatchStages] = {};
        const int64_t n = p.n;
        if (n > 0) {
            if (p.transport) {
                blocks[kStVertices] = vertex_launch_blocks(in.surface.vertex_count, host.vertex_block);
                blocks[kStOwners] = owner_blocks(in.surface.owner_count, n);
                blocks[kStScatter] = blocks_for(n, kThreads);
            }
            // node-box passes: about one block per 2048 particles (256 nodes at 8 particles a cell)
            const uint32_t box = (uint32_t)std::min<int64_t>(std::max<int64_t>(1, (n + 2047) / 2048), 4 * sms);
            if (p.transport) blocks[kStDiffuse] = box;
            blocks[kStClear] = box;
            blocks[kStP2G] = blocks_for(n, kThreads);
            blocks[kStGrid] = box;
            if (surrogate) {
                // a persistent share of 4 CTAs per SM in proportion to the particles
                const int64_t share = std::max<int64_t>(1, (int64_t)(4.0 * sms * (double)n / (double)particles + 0.5));
                blocks[kStSurrogate] = (uint32_t)std::min<int64_t>(share, blocks_for(n, 128));
            } else {
                blocks[kStG2P] = blocks_for(n, 128);
            }
        }
        for (int st = 0; st < kBatchStages; ++st) {
            uint32_t* f = first.data() + (size_t)st * (count + 1);
            BK_REQUIRE((uint64_t)f[k] + blocks[st] < (1ull << 31), "bk_batch_create: too many blocks in one stage");
            f[k + 1] = f[k] + blocks[st];
        }
    }
    std::vector<int32_t> owner;
    for (int st = 0; st < kBatchStages; ++st) {
        host.total[st] = first[(size_t)st * (count + 1) + count];
        host.owner_offset[st] = (uint32_t)owner.size();
        for (int k = 0; k < count; ++k)
            owner.insert(owner.end(), first[(size_t)st * (count + 1) + k + 1] - first[(size_t)st * (count + 1) + k], k);
    }
    BK_REQUIRE(owner.size() < (1ull << 31), "bk_batch_create: too many blocks");
    if (owner.empty()) owner.push_back(0);
    BkBatch* out = new BkBatch(host);
    if (cudaMalloc(&out->entries, entries.size() * sizeof(BatchEntry)) != cudaSuccess ||
        cudaMalloc(&out->first, first.size() * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&out->owner, owner.size() * sizeof(int32_t)) != cudaSuccess) {
        cudaFree(out->entries);
        cudaFree(out->first);
        cudaFree(out->owner);
        delete out;
        cudaGetLastError();
        return fail(BK_ERR_LAUNCH, "bk_batch_create: device allocation failed");
    }
    if (cudaMemcpy(out->entries, entries.data(), entries.size() * sizeof(BatchEntry), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(out->first, first.data(), first.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(out->owner, owner.data(), owner.size() * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess) {
        bk_batch_destroy(out);
        return fail(BK_ERR_LAUNCH, "bk_batch_create: table upload failed");
    }
    *batch = out;
    return BK_OK;
}

int bk_batch_substep(BkBatch* batch, int32_t parity, int32_t phases, int32_t prescattered, int32_t prescatter_next,
                     void* stream) {
    BK_REQUIRE(batch && (parity == 0 || parity == 1), "bk_batch_substep: bad batch or parity");
    BK_REQUIRE(!prescatter_next || (phases & BK_PHASE_MECHANICS),
               "bk_batch_substep: the transport prescatter runs in the G2P kernel of a mechanics phase");
    const BkBatch& B = *batch;
    BatchArgs a{};
    a.entries = B.entries;
    a.first = B.first;
    a.owner = B.owner;
    for (int st = 0; st < kBatchStages; ++st) a.owner_offset[st] = B.owner_offset[st];
    a.count = B.count;
    a.parity = parity;
    a.prescattered = prescattered ? 1 : 0;
    a.prescatter_next = prescatter_next ? 1 : 0;
    const uint32_t* T = B.total;
    cudaStream_t s = S(stream);
    if ((phases & BK_PHASE_TRANSPORT) && B.any_transport) {
        if (T[kStVertices]) {
            int rec = profile_begin("batch_surface_vertices", s);
            switch (B.vertex_block) {
                case 256: kb_surface_vertices<256><<<T[kStVertices], 256, 0, s>>>(a); break;
                case 128: kb_surface_vertices<128><<<T[kStVertices], 128, 0, s>>>(a); break;
                default: kb_surface_vertices<32><<<T[kStVertices], vertex_launch_threads(32), 0, s>>>(a); break;
            }
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/surface_vertices")) return rc;
        }
        if (T[kStOwners]) {
            int rec = profile_begin("batch_surface_owners", s);
            kb_surface_owners<<<T[kStOwners], kOwnerThreads, 0, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/surface_owners")) return rc;
        }
        if (T[kStScatter] && !(prescattered && B.all_prescatter)) {
            int rec = profile_begin("batch_transport_scatter", s);
            kb_transport_scatter<<<T[kStScatter], kThreads, 0, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/transport_scatter")) return rc;
        }
        if (T[kStDiffuse]) {
            int rec = profile_begin("batch_diffuse", s);
            kb_diffuse<<<T[kStDiffuse], kDiffThreads, 0, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/diffuse")) return rc;
        }
    }
    if (phases & BK_PHASE_MECHANICS) {
        if (T[kStClear]) {
            int rec = profile_begin("batch_clear_previous", s);
            kb_clear_previous<<<T[kStClear], kThreads, 0, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/clear_previous")) return rc;
        }
        if (T[kStP2G]) {
            int rec = profile_begin("batch_p2g", s);
            if (int rc = allow_smem(B.staged ? (const void*)kb_p2g<true> : (const void*)kb_p2g<false>,
                                    kP2GSmemBytes, "bk_batch_substep/p2g"))
                return rc;
            if (B.staged) kb_p2g<true><<<T[kStP2G], kThreads, kP2GSmemBytes, s>>>(a);
            else kb_p2g<false><<<T[kStP2G], kThreads, kP2GSmemBytes, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/p2g")) return rc;
        }
        if (T[kStGrid]) {
            int rec = profile_begin("batch_grid_update", s);
            kb_grid_update<<<T[kStGrid], kThreads, 0, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/grid_update")) return rc;
        }
        if (T[kStG2P]) {
            int rec = profile_begin("batch_g2p_return", s);
            const size_t smem = prescatter_next ? sizeof(G2PTransportTile) : 0;
            kb_g2p_return<<<T[kStG2P], 128, smem, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/g2p_return")) return rc;
        }
        if (T[kStSurrogate]) {
            int rec = profile_begin("batch_g2p_return_surrogate", s);
            kb_g2p_return_surrogate<<<T[kStSurrogate], 128, 0, s>>>(a);
            profile_end(rec, s);
            if (int rc = check_launch("bk_batch_substep/g2p_return_surrogate")) return rc;
        }
    }
    return BK_OK;
}

int bk_batch_destroy(BkBatch* batch) {
    if (!batch) return BK_OK;
    cudaFree(batch->entries);
    cudaFree(batch->first);
    cudaFree(batch->owner);
    delete batch;
    return BK_OK;
}

}  // extern "C"
