// Return-map surrogate MLP (7 -> 64 -> 64 -> 3, SiLU) on the 5th-generation tensor cores.
//
// One CTA evaluates a tile of 128 rows (one row per thread, 4 warps): each layer's input is
// written by its row's thread into shared memory as BF16 in the canonical K-major layout without
// swizzle, one elected thread issues tcgen05.mma (M = 128, kind::f16, BF16 x BF16 -> FP32) with
// the packed weights as the B operand, the accumulator lands in tensor memory, and every warp
// reads back its own 32 rows with tcgen05.ld (TMEM lane = row = thread) to add the FP32 bias and
// apply SiLU before writing the next layer's input. 64 TMEM columns are reused by the three layers.
//
// Canonical K-major layout (no swizzle): 8x16-byte core matrices; element (row, k) of an operand
// with K columns sits at byte (row / 8) * SBO + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2 with
// SBO = K * 16 (leading-dimension offset 128 bytes between the two core matrices of one K = 16 step).
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace bk {
namespace mlp {

constexpr int kRows = 128;       // rows per tile (M)
constexpr int kIn = 16;          // padded input width (7 features)
constexpr int kHidden = 64;
constexpr int kOut = 16;         // padded output width (3 outputs)
constexpr int kFeatures = 7;
constexpr int kOutputs = 3;
constexpr int kTmemCols = 64;

// Packed weight blob (bytes): BF16 W1^T (64 x 16), W2^T (64 x 64), W3^T (16 x 64) in the canonical
// layout above, then FP32 biases b1[64], b2[64], b3[16].
constexpr int kW1Offset = 0;
constexpr int kW2Offset = kW1Offset + kHidden * kIn * 2;        // 2048
constexpr int kW3Offset = kW2Offset + kHidden * kHidden * 2;    // 10240
constexpr int kB1Offset = kW3Offset + kOut * kHidden * 2;       // 12288
constexpr int kB2Offset = kB1Offset + kHidden * 4;              // 12544
constexpr int kB3Offset = kB2Offset + kHidden * 4;              // 12800
constexpr int kBlobBytes = kB3Offset + kOut * 4;                // 12864
constexpr int kActBytes = kRows * kHidden * 2;                  // 16384: one BF16 activation tile

// Byte offset of element (row, k) in a K-major operand with `K` columns.
__host__ __device__ constexpr int operand_offset(int row, int k, int K) {
    return (row / 8) * (K * 16) + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2;
}

// Shared-memory matrix descriptor (sm100): start address, leading/stride byte offsets (>> 4),
// descriptor version 1 at bit 46, no swizzle (layout type 0 in bits 61..63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor for kind::f16: FP32 accumulate (bits 4-5 = 1), BF16 A and B (bits 7-9 and
// 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Make this thread's generic-proxy shared-memory writes visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar_smem) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_smem)
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar_smem, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar_smem), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for the mbarrier phase with parity `parity`; gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar_smem, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar_smem), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// SiLU for the inference epilogue: z * sigmoid(z) = z/2 (1 + tanh(z/2)) with the hardware tanh
// approximation (one instruction; relative error ~2^-11, below the BF16 rounding of the result).
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float silu(float z) { return 0.5f * z * (1.0f + tanh_approx(0.5f * z)); }

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // .x = a (low half), .y = b
    return *reinterpret_cast<uint32_t*>(&h);
}

// Write 8 consecutive K-values (one 16-byte core-matrix row) of `row`, starting at k0 (multiple of 8).
__device__ __forceinline__ void store_row8(unsigned char* tile, int row, int k0, int K, const float* v) {
    uint4 q;
    q.x = pack_bf16x2(v[0], v[1]);
    q.y = pack_bf16x2(v[2], v[3]);
    q.z = pack_bf16x2(v[4], v[5]);
    q.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4*>(tile + operand_offset(row, k0, K)) = q;
}

// Shared memory of one tile evaluation. `act` holds the BF16 layer inputs; `blob` the packed weights.
struct TileSmem {
    alignas(128) unsigned char act[kActBytes];
    alignas(128) unsigned char blob[kBlobBytes];
    alignas(8) uint64_t mbar;
    uint32_t tmem_base;
    int32_t failed;
};

// Copy the packed weights into shared memory (all threads), initialise the mbarrier and allocate
// TMEM (warp 0). Ends with a block barrier.
__device__ __forceinline__ void tile_setup(TileSmem& s, const unsigned char* __restrict__ blob) {
    const int t = threadIdx.x;
    const uint4* src = reinterpret_cast<const uint4*>(blob);
    uint4* dst = reinterpret_cast<uint4*>(s.blob);
    for (int k = t; k < kBlobBytes / 16; k += blockDim.x) dst[k] = __ldg(src + k);
    if (t == 0) {
        mbar_init(smem_addr(&s.mbar), 1);
        s.failed = 0;
    }
    if (t < 32) tmem_alloc(smem_addr(&s.tmem_base), kTmemCols);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

__device__ __forceinline__ void tile_teardown(TileSmem& s) {
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (threadIdx.x < 32) tmem_dealloc(s.tmem_base, kTmemCols);
}

// One layer: D[128 x N] = act[128 x K] * W^T, with W^T (N x K) at blob offset `w_off`. Issued by
// thread 0; all threads wait for completion. Returns false if the wait gave up.
__device__ __forceinline__ bool tile_layer(TileSmem& s, int w_off, int K, int N, uint32_t phase) {
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (threadIdx.x == 0) {
        const uint32_t a0 = smem_addr(s.act), b0 = smem_addr(s.blob + w_off);
        const uint32_t idesc = instr_desc_bf16(kRows, N);
        for (int k = 0; k < K / 16; ++k) {
            uint64_t ad = smem_desc(a0 + k * 256, 128, K * 16);
            uint64_t bd = smem_desc(b0 + k * 256, 128, K * 16);
            mma_bf16(s.tmem_base, ad, bd, idesc, k > 0 ? 1u : 0u);
        }
        mma_commit(smem_addr(&s.mbar));
    }
    bool ok = mbar_wait(smem_addr(&s.mbar), phase & 1u, 1u << 20);
    if (!ok) s.failed = 1;
    fence_after_sync();
    return ok;
}

// Evaluate the tile. `x` is this thread's normalised input row (kFeatures values; ignored when
// `active` is false, which writes a zero row). On return `y` holds the kOutputs outputs. `phase`
// counts the mbarrier completions of this CTA (3 per call). Returns false if a tensor-core wait
// gave up (outputs then undefined; the caller falls back).
__device__ inline bool tile_eval(TileSmem& s, const float* x, bool active, float* y, uint32_t& phase) {
    const int row = threadIdx.x;
    const uint32_t lane_base = s.tmem_base + ((uint32_t)(row & ~31) << 16);
    {
        // Layer-1 input (K = 16): the BF16 inputs in columns 0-6 and their BF16 remainders
        // x - bf16(x) in columns 8-14, which the packed W1 multiplies by the same weights, so the
        // first layer sees each input to ~16 significant bits instead of BF16's 8.
        float v[8], r[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float xk = (active && k < kFeatures) ? x[k] : 0.0f;
            v[k] = __bfloat162float(__float2bfloat16_rn(xk));
            r[k] = xk - v[k];
        }
        store_row8(s.act, row, 0, kIn, v);
        store_row8(s.act, row, 8, kIn, r);
    }
    bool ok = tile_layer(s, kW1Offset, kIn, kHidden, phase++);
    const float* b1 = reinterpret_cast<const float*>(s.blob + kB1Offset);
    const float* b2 = reinterpret_cast<const float*>(s.blob + kB2Offset);
    const float* b3 = reinterpret_cast<const float*>(s.blob + kB3Offset);
    // Layer 1 epilogue: h1 = SiLU(acc + b1) -> BF16 layer-2 input (K = 64). The MMA has finished
    // reading act, so it is overwritten in place.
#pragma unroll
    for (int c = 0; c < kHidden; c += 16) {
        float v[16];
        tmem_ld16(lane_base + c, v);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = silu(v[k] + b1[c + k]);
        store_row8(s.act, row, c, kHidden, v);
        store_row8(s.act, row, c + 8, kHidden, v + 8);
    }
    ok = tile_layer(s, kW2Offset, kHidden, kHidden, phase++) && ok;
#pragma unroll
    for (int c = 0; c < kHidden; c += 16) {
        float v[16];
        tmem_ld16(lane_base + c, v);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = silu(v[k] + b2[c + k]);
        store_row8(s.act, row, c, kHidden, v);
        store_row8(s.act, row, c + 8, kHidden, v + 8);
    }
    ok = tile_layer(s, kW3Offset, kHidden, kOut, phase++) && ok;
    {
        float v[16];
        tmem_ld16(lane_base, v);
#pragma unroll
        for (int k = 0; k < kOutputs; ++k) y[k] = v[k] + b3[k];
    }
    return ok;
}

}  // namespace mlp
}  // namespace bk
