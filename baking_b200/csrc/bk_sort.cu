// Particle reordering by grid cell: the permutation that makes particles sharing a quadratic
// stencil base (floor((x - origin)/dx - 0.5), the base every transfer kernel computes)
// consecutive, with the bases in Morton order. The scatter kernels (P2G, the transport scatter
// and their adjoints) sum each warp's runs of equal base in registers and stage a block's node box
// in shared memory, so both the run length and the box size follow from this order.
//
// One key kernel (interleaved base bits; stencils leaving the grid and non-finite positions get
// the largest key) and a stable least-significant-digit radix sort over 3 x ceil(log2 R) key bits
// (CUB's DeviceRadixSort::SortPairs), particle index as the value: particles of one cell keep
// their relative order.
#include <algorithm>
#include <cstdint>
#include <cub/device/device_radix_sort.cuh>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_device.cuh"

using namespace bk;

namespace {

constexpr int kThreads = 256;

int key_bits(int32_t resolution) {
    int bits = 1;
    while ((1 << bits) < resolution) ++bits;
    return bits;
}

// Spread the low 21 bits of v so that bit k lands on bit 3k.
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

struct SortGeometry {
    float origin[3];
    float dx;
    int R;
    uint64_t invalid_key;
};

__global__ void __launch_bounds__(kThreads) k_cell_keys(int64_t n, const float* __restrict__ x, int64_t pitch,
                                                        SortGeometry geo, uint64_t* __restrict__ keys,
                                                        int32_t* __restrict__ values) {
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    if (i >= n) return;
    const V3 p = load_v3(x, i, pitch);
    const Stencil st = make_stencil(p, geo.origin, geo.dx, geo.R);
    uint64_t key = geo.invalid_key;
    if (st.valid && isfinite(p.v[0]) && isfinite(p.v[1]) && isfinite(p.v[2]))
        key = spread3((uint64_t)st.b[2]) | (spread3((uint64_t)st.b[1]) << 1) | (spread3((uint64_t)st.b[0]) << 2);
    keys[i] = key;
    values[i] = (int32_t)i;
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Bytes of CUB's temporary storage for n pairs, or 0 with an error recorded.
size_t cub_bytes(int64_t n, int end_bit) {
    size_t bytes = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                                    (const int32_t*)nullptr, (int32_t*)nullptr, (int)n, 0, end_bit);
    if (e != cudaSuccess) {
        fail(BK_ERR_LAUNCH, cudaGetErrorString(e));
        return 0;
    }
    return bytes;
}

// A group of per-particle arrays permuted together: each array's planes gathered into its slice of
// the scratch buffer (element k of plane p <- element order[k]), then copied back in order. One
// launch per pass for the whole group; block row y is the array, block column x a range of
// particles, each thread one particle and every plane of the array (order[k] read once).
constexpr int kPermuteGroupMax = 64;
struct PermuteEntry {
    void* data;
    int64_t pitch;
    int64_t offset;  // bytes into the scratch buffer (256-byte aligned)
    int32_t planes, bytes;
};
struct PermuteGroup {
    PermuteEntry e[kPermuteGroupMax];
};

template <bool kBack, class T>
__device__ __forceinline__ void permute_planes(int64_t n, int64_t k, int64_t src, const PermuteEntry& E,
                                               unsigned char* scratch) {
    T* d = static_cast<T*>(E.data);
    T* sc = reinterpret_cast<T*>(scratch + E.offset);
    for (int p = 0; p < E.planes; ++p) {
        if constexpr (kBack) d[p * E.pitch + k] = sc[p * n + k];
        else sc[p * n + k] = d[p * E.pitch + src];
    }
}

template <bool kBack>
__global__ void __launch_bounds__(kThreads) k_permute_group(int64_t n, const int32_t* __restrict__ order,
                                                            const __grid_constant__ PermuteGroup g,
                                                            unsigned char* __restrict__ scratch) {
    const PermuteEntry& E = g.e[blockIdx.y];
    for (int64_t k = blockIdx.x * (int64_t)kThreads + threadIdx.x; k < n; k += (int64_t)gridDim.x * kThreads) {
        const int64_t src = kBack ? k : (int64_t)order[k];
        if (E.bytes == 4) permute_planes<kBack, uint32_t>(n, k, src, E, scratch);
        else permute_planes<kBack, uint64_t>(n, k, src, E, scratch);
    }
}

}  // namespace

extern "C" {

int64_t bk_sort_by_cell_scratch_bytes(int64_t n, int32_t resolution) {
    if (n < 0 || n > INT32_MAX || resolution < 4 || resolution >= (1 << 20)) {
        fail(BK_ERR_ARGUMENT, "bk_sort_by_cell_scratch_bytes: bad particle count or resolution");
        return -1;
    }
    if (n == 0) return 0;
    const size_t cub = cub_bytes(n, 3 * key_bits(resolution));
    if (cub == 0) return -1;
    return (int64_t)(2 * align256(8 * (size_t)n) + align256(4 * (size_t)n) + cub);
}

int bk_sort_by_cell(int64_t n, int64_t pitch, const float* x, const float* origin, float dx, int32_t resolution,
                    int32_t* order, void* scratch, int64_t scratch_bytes, void* stream) {
    if (n < 0 || n > INT32_MAX || pitch < n || resolution < 4 || resolution >= (1 << 20) || !(dx > 0.0f))
        return fail(BK_ERR_ARGUMENT, "bk_sort_by_cell: bad particle count, pitch, resolution or spacing");
    if (n == 0) return BK_OK;
    if (!x || !origin || !order || !scratch) return fail(BK_ERR_ARGUMENT, "bk_sort_by_cell: null argument");
    if (((uintptr_t)scratch & 255) != 0) return fail(BK_ERR_ARGUMENT, "bk_sort_by_cell: scratch not 256-byte aligned");
    const int end_bit = 3 * key_bits(resolution);
    const size_t cub = cub_bytes(n, end_bit);
    if (cub == 0) return BK_ERR_LAUNCH;
    const size_t key_bytes = align256(8 * (size_t)n), value_bytes = align256(4 * (size_t)n);
    if (scratch_bytes < (int64_t)(2 * key_bytes + value_bytes + cub))
        return fail(BK_ERR_ARGUMENT, "bk_sort_by_cell: scratch smaller than bk_sort_by_cell_scratch_bytes");
    char* base = static_cast<char*>(scratch);
    uint64_t* keys_in = reinterpret_cast<uint64_t*>(base);
    uint64_t* keys_out = reinterpret_cast<uint64_t*>(base + key_bytes);
    int32_t* values_in = reinterpret_cast<int32_t*>(base + 2 * key_bytes);
    void* temp = base + 2 * key_bytes + value_bytes;
    SortGeometry geo;
    for (int a = 0; a < 3; ++a) geo.origin[a] = origin[a];
    geo.dx = dx;
    geo.R = resolution;
    geo.invalid_key = end_bit >= 64 ? ~0ull : ((1ull << end_bit) - 1);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_cell_keys<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(n, x, pitch, geo, keys_in, values_in);
    if (int rc = check_launch("bk_sort_by_cell/keys")) return rc;
    size_t temp_bytes = cub;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys_in, keys_out, values_in, order, (int)n, 0,
                                                    end_bit, s);
    if (e != cudaSuccess) return fail(BK_ERR_LAUNCH, cudaGetErrorString(e));
    return check_launch("bk_sort_by_cell/radix_sort");
}

int bk_permute_particles(int64_t n, const int32_t* order, int32_t array_count, const BkParticleArray* arrays,
                         void* scratch, int64_t scratch_bytes, void* stream) {
    if (n < 0 || array_count < 0) return fail(BK_ERR_ARGUMENT, "bk_permute_particles: negative count");
    if (n > INT32_MAX) return fail(BK_ERR_ARGUMENT, "bk_permute_particles: more particles than an int32 order can index");
    if (n == 0 || array_count == 0) return BK_OK;
    if (!order || !arrays || !scratch) return fail(BK_ERR_ARGUMENT, "bk_permute_particles: null argument");
    if (((uintptr_t)scratch & 255) != 0) return fail(BK_ERR_ARGUMENT, "bk_permute_particles: scratch not 256-byte aligned");
    for (int32_t a = 0; a < array_count; ++a) {
        const BkParticleArray& arr = arrays[a];
        if (!arr.data || arr.planes < 1 || arr.pitch < n || (arr.element_bytes != 4 && arr.element_bytes != 8))
            return fail(BK_ERR_ARGUMENT, "bk_permute_particles: bad array (data, planes, pitch or element size)");
        if (((uintptr_t)arr.data & (uintptr_t)(arr.element_bytes - 1)) != 0)
            return fail(BK_ERR_ARGUMENT, "bk_permute_particles: array not aligned to its element size");
        if ((int64_t)arr.planes * n * arr.element_bytes > scratch_bytes)
            return fail(BK_ERR_ARGUMENT, "bk_permute_particles: scratch smaller than the largest array");
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = static_cast<unsigned char*>(scratch);
    const unsigned blocks = (unsigned)std::min<int64_t>((n + kThreads - 1) / kThreads, 2048);
    // Groups of consecutive arrays whose slices (each rounded up to 256 bytes) fit the scratch
    // buffer and the launch table; a group is gathered, then copied back, before the next starts.
    int32_t a = 0;
    while (a < array_count) {
        PermuteGroup g;
        int count = 0;
        int64_t used = 0;
        while (a < array_count && count < kPermuteGroupMax) {
            const BkParticleArray& arr = arrays[a];
            const int64_t bytes = ((int64_t)arr.planes * n * arr.element_bytes + 255) & ~(int64_t)255;
            if (count > 0 && used + bytes > scratch_bytes) break;
            g.e[count] = PermuteEntry{arr.data, arr.pitch, used, arr.planes, arr.element_bytes};
            used += bytes;
            ++count;
            ++a;
        }
        const dim3 grid(blocks, (unsigned)count);
        k_permute_group<false><<<grid, kThreads, 0, s>>>(n, order, g, base);
        if (int rc = check_launch("bk_permute_particles/gather")) return rc;
        k_permute_group<true><<<grid, kThreads, 0, s>>>(n, order, g, base);
        if (int rc = check_launch("bk_permute_particles/copy_back")) return rc;
    }
    return BK_OK;
}

}  // extern "C"
