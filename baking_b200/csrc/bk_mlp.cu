// Return-map surrogate: stand-alone tensor-core inference, the fused training kernels (forward +
// backward on the CUDA cores with the inference's BF16 rounding, FP32 accumulation), Adam, and the
// packing of the FP32 master weights into the tensor-core operand layout.
//
// Parameter vector (FP32 master weights, in x out row-major):
//   W1 [7][64] | b1 [64] | W2 [64][64] | b2 [64] | W3 [64][3] | b3 [3]
// Normalisation: x = (feature - in_mean) / in_scale per feature, outputs y are in units of
// out_scale (prediction = y * out_scale).
#include <cstdio>

#include "baking_b200.h"
#include "bk_common.h"
#include "bk_mlp.cuh"

using namespace bk;
using namespace bk::mlp;

namespace {

constexpr int kP_W1 = 0;
constexpr int kP_B1 = kP_W1 + kFeatures * kHidden;   // 448
constexpr int kP_W2 = kP_B1 + kHidden;                // 512
constexpr int kP_B2 = kP_W2 + kHidden * kHidden;      // 4608
constexpr int kP_W3 = kP_B2 + kHidden;                // 4672
constexpr int kP_B3 = kP_W3 + kHidden * kOutputs;     // 4864
constexpr int kParamCount = kP_B3 + kOutputs;         // 4867
static_assert(kParamCount == BK_MLP_PARAMS, "parameter count mismatch");

struct Norm {
    float in_mean[8], in_scale[8], out_scale[4];
};

Norm to_norm(const BkMlpNorm& n) {
    Norm o;
    for (int k = 0; k < 8; ++k) { o.in_mean[k] = n.in_mean[k]; o.in_scale[k] = n.in_scale[k]; }
    for (int k = 0; k < 4; ++k) o.out_scale[k] = n.out_scale[k];
    return o;
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + __expf(-z)); }

// ------------------------------------------------------------------ inference
__global__ void __launch_bounds__(kRows) k_mlp_infer(int64_t n, const float* __restrict__ features, Norm nm,
                                                     const unsigned char* __restrict__ blob, float* __restrict__ out,
                                                     int32_t* __restrict__ status) {
    __shared__ TileSmem s;
    tile_setup(s, blob);
    uint32_t phase = 0;
    for (int64_t base = (int64_t)blockIdx.x * kRows; base < n; base += (int64_t)gridDim.x * kRows) {
        const int64_t i = base + threadIdx.x;
        const bool active = i < n;
        float x[kFeatures];
#pragma unroll
        for (int k = 0; k < kFeatures; ++k) x[k] = active ? (features[i * 8 + k] - nm.in_mean[k]) / nm.in_scale[k] : 0.f;
        float y[kOutputs];
        bool ok = tile_eval(s, x, active, y, phase);
        if (active && ok) {
#pragma unroll
            for (int k = 0; k < kOutputs; ++k) out[i * 4 + k] = y[k] * nm.out_scale[k];
            out[i * 4 + 3] = 0.f;
        }
        __syncthreads();
        if (s.failed) {  // uniform across the block: a tensor-core wait gave up
            if (threadIdx.x == 0) atomicExch(status, 1);
            break;
        }
    }
    tile_teardown(s);
}

// ------------------------------------------------------------------- training
// One block = one tile of 128 samples, one sample per thread. Per-sample activations live in
// shared memory in feature-major rows of kStride floats (padded so that a warp reading one feature
// of 32 samples, or 32 features of one sample, hits distinct banks).
constexpr int kStride = kRows + 1;

struct GradSmem {
    float W1[kFeatures * kHidden], W2[kHidden * kHidden], W3[kHidden * kOutputs];
    float b1[kHidden], b2[kHidden], b3[kOutputs];
    float X[kFeatures * kStride];
    float H1[kHidden * kStride], D1[kHidden * kStride], H2[kHidden * kStride], D2[kHidden * kStride];
    float DY[kOutputs * kStride];
    float loss[kRows / 32];
};

__global__ void __launch_bounds__(kRows) k_mlp_grad(int64_t batch, const float* __restrict__ features,
                                                    const float* __restrict__ targets, Norm nm,
                                                    const float* __restrict__ params, float* __restrict__ grads,
                                                    double* __restrict__ loss_sum) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    GradSmem& s = *reinterpret_cast<GradSmem*>(smem_raw);
    const int t = threadIdx.x;
    // Weights as the tensor cores see them (BF16), biases in FP32.
    for (int k = t; k < kFeatures * kHidden; k += kRows) s.W1[k] = bf16_round(params[kP_W1 + k]);
    for (int k = t; k < kHidden * kHidden; k += kRows) s.W2[k] = bf16_round(params[kP_W2 + k]);
    for (int k = t; k < kHidden * kOutputs; k += kRows) s.W3[k] = bf16_round(params[kP_W3 + k]);
    if (t < kHidden) { s.b1[t] = params[kP_B1 + t]; s.b2[t] = params[kP_B2 + t]; }
    if (t < kOutputs) s.b3[t] = params[kP_B3 + t];
    const int64_t i = (int64_t)blockIdx.x * kRows + t;
    const bool active = i < batch;
    const float inv_count = 1.0f / (float)(batch * kOutputs);
    for (int k = 0; k < kFeatures; ++k) {
        // the inference's two-term BF16 input: bf16(x) + bf16(x - bf16(x))
        const float x = active ? (features[i * 8 + k] - nm.in_mean[k]) / nm.in_scale[k] : 0.f;
        const float hi = bf16_round(x);
        s.X[k * kStride + t] = hi + bf16_round(x - hi);
    }
    __syncthreads();
    // forward: layer 1
    for (int j = 0; j < kHidden; ++j) {
        float z = s.b1[j];
#pragma unroll
        for (int k = 0; k < kFeatures; ++k) z = fmaf(s.X[k * kStride + t], s.W1[k * kHidden + j], z);
        float sg = sigmoid(z);
        s.H1[j * kStride + t] = bf16_round(z * sg);
        s.D1[j * kStride + t] = sg * (1.0f + z * (1.0f - sg));
    }
    // layer 2
    for (int j = 0; j < kHidden; ++j) {
        float z = s.b2[j];
#pragma unroll 8
        for (int k = 0; k < kHidden; ++k) z = fmaf(s.H1[k * kStride + t], s.W2[k * kHidden + j], z);
        float sg = sigmoid(z);
        s.H2[j * kStride + t] = bf16_round(z * sg);
        s.D2[j * kStride + t] = sg * (1.0f + z * (1.0f - sg));
    }
    // layer 3 + loss
    float sq = 0.f;
#pragma unroll
    for (int o = 0; o < kOutputs; ++o) {
        float y = s.b3[o];
        for (int k = 0; k < kHidden; ++k) y = fmaf(s.H2[k * kStride + t], s.W3[k * kOutputs + o], y);
        float d = active ? y - targets[i * 4 + o] / nm.out_scale[o] : 0.f;
        sq += d * d;
        s.DY[o * kStride + t] = 2.0f * d * inv_count;
    }
    // backward to layer-2 pre-activations: dz2 = (W3 dy) * silu'(z2), in place of D2
    for (int j = 0; j < kHidden; ++j) {
        float g = 0.f;
#pragma unroll
        for (int o = 0; o < kOutputs; ++o) g = fmaf(s.W3[j * kOutputs + o], s.DY[o * kStride + t], g);
        s.D2[j * kStride + t] *= g;
    }
    __syncthreads();
    // dz1 = (W2 dz2) * silu'(z1), in place of D1 (each thread its own sample: no race with D2 reads)
    for (int k = 0; k < kHidden; ++k) {
        float g = 0.f;
#pragma unroll 8
        for (int j = 0; j < kHidden; ++j) g = fmaf(s.W2[k * kHidden + j], s.D2[j * kStride + t], g);
        s.D1[k * kStride + t] *= g;
    }
    __syncthreads();
    // weight gradients: sums over the tile's samples, then one atomic per parameter per block
    // dW2[k][j] = sum_b H1[k][b] dz2[j][b]: thread t owns k = t / 2, j in [32 (t % 2), +32)
    {
        const int k = t >> 1, j0 = (t & 1) * 32;
        float acc[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) acc[q] = 0.f;
        for (int b = 0; b < kRows; ++b) {
            float h = s.H1[k * kStride + b];
#pragma unroll
            for (int q = 0; q < 32; ++q) acc[q] = fmaf(h, s.D2[(j0 + q) * kStride + b], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < 32; ++q) atomicAdd(grads + kP_W2 + k * kHidden + j0 + q, acc[q]);
    }
    // dW1[k][j] = sum_b X[k][b] dz1[j][b] (7 x 64), db1, db2 (thread j < 64)
    if (t < kHidden) {
        const int j = t;
        float a[kFeatures] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        float g1 = 0.f, g2 = 0.f;
        for (int b = 0; b < kRows; ++b) {
            float d1 = s.D1[j * kStride + b];
#pragma unroll
            for (int k = 0; k < kFeatures; ++k) a[k] = fmaf(s.X[k * kStride + b], d1, a[k]);
            g1 += d1;
            g2 += s.D2[j * kStride + b];
        }
#pragma unroll
        for (int k = 0; k < kFeatures; ++k) atomicAdd(grads + kP_W1 + k * kHidden + j, a[k]);
        atomicAdd(grads + kP_B1 + j, g1);
        atomicAdd(grads + kP_B2 + j, g2);
    } else {
        // dW3[k][o] = sum_b H2[k][b] dy[o][b] (64 x 3), db3: threads 64..127 own k = t - 64
        const int k = t - kHidden;
        float a[kOutputs] = {0.f, 0.f, 0.f};
        for (int b = 0; b < kRows; ++b) {
            float h = s.H2[k * kStride + b];
#pragma unroll
            for (int o = 0; o < kOutputs; ++o) a[o] = fmaf(h, s.DY[o * kStride + b], a[o]);
        }
#pragma unroll
        for (int o = 0; o < kOutputs; ++o) atomicAdd(grads + kP_W3 + k * kOutputs + o, a[o]);
        if (k < kOutputs) {
            float g = 0.f;
            for (int b = 0; b < kRows; ++b) g += s.DY[k * kStride + b];
            atomicAdd(grads + kP_B3 + k, g);
        }
    }
    // loss
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if ((t & 31) == 0) s.loss[t >> 5] = sq;
    __syncthreads();
    if (t == 0 && loss_sum) {
        float tot = 0.f;
        for (int w = 0; w < kRows / 32; ++w) tot += s.loss[w];
        atomicAdd(loss_sum, (double)tot);
    }
}

__global__ void k_mlp_adam(int count, float* __restrict__ params, const float* __restrict__ grads,
                           float* __restrict__ m, float* __restrict__ v, float lr, float beta1, float beta2,
                           float eps, float c1, float c2) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    float g = grads[k];
    float mk = beta1 * m[k] + (1.0f - beta1) * g;
    float vk = beta2 * v[k] + (1.0f - beta2) * g * g;
    m[k] = mk;
    v[k] = vk;
    params[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// FP32 master weights -> BF16 operands in the canonical layout + FP32 biases (zero padding).
__global__ void k_mlp_pack(const float* __restrict__ params, unsigned char* __restrict__ blob) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    auto put = [&](int off, float x) { *reinterpret_cast<__nv_bfloat16*>(blob + off) = __float2bfloat16_rn(x); };
    if (t < kHidden * kIn) {  // W1^T: n x k (64 x 16)
        int n = t / kIn, k = t % kIn;
        // Columns 0-6 multiply the BF16 inputs, columns 8-14 the BF16 remainders x - bf16(x) of the
        // same inputs (tile_eval): the same weights, so the layer sees x to ~16 bits, not 8.
        const int f = k < kFeatures ? k : (k >= 8 && k < 8 + kFeatures ? k - 8 : -1);
        put(kW1Offset + operand_offset(n, k, kIn), f >= 0 ? params[kP_W1 + f * kHidden + n] : 0.f);
    }
    if (t < kHidden * kHidden) {  // W2^T: 64 x 64
        int n = t / kHidden, k = t % kHidden;
        put(kW2Offset + operand_offset(n, k, kHidden), params[kP_W2 + k * kHidden + n]);
    }
    if (t < kOut * kHidden) {  // W3^T: 16 x 64
        int n = t / kHidden, k = t % kHidden;
        put(kW3Offset + operand_offset(n, k, kHidden), n < kOutputs ? params[kP_W3 + k * kOutputs + n] : 0.f);
    }
    float* b = reinterpret_cast<float*>(blob + kB1Offset);
    if (t < kHidden) { b[t] = params[kP_B1 + t]; b[kHidden + t] = params[kP_B2 + t]; }
    if (t < kOut) b[2 * kHidden + t] = t < kOutputs ? params[kP_B3 + t] : 0.f;
}

}  // namespace

extern "C" {

int bk_mlp_infer(int64_t n, const float* features, const BkMlpNorm* norm, const void* packed, float* outputs,
                 int32_t* status, void* stream) {
    if (n < 0 || (n > 0 && (!features || !norm || !packed || !outputs || !status)))
        return fail(BK_ERR_ARGUMENT, "bk_mlp_infer: null argument");
    if (reinterpret_cast<uintptr_t>(packed) % 16 != 0) return fail(BK_ERR_ARGUMENT, "bk_mlp_infer: packed weights must be 16-byte aligned");
    if (n == 0) return BK_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int64_t tiles = (n + kRows - 1) / kRows;
    unsigned grid = (unsigned)(tiles < 148 * 4 ? tiles : 148 * 4);
    k_mlp_infer<<<grid, kRows, 0, s>>>(n, features, to_norm(*norm), static_cast<const unsigned char*>(packed),
                                       outputs, status);
    return check_launch("bk_mlp_infer");
}

int bk_mlp_gradient(int64_t batch, const float* features, const float* targets, const BkMlpNorm* norm,
                    const float* params, float* grads, double* loss_sum, void* stream) {
    if (batch < 0 || (batch > 0 && (!features || !targets || !norm || !params || !grads)))
        return fail(BK_ERR_ARGUMENT, "bk_mlp_gradient: null argument");
    if (batch == 0) return BK_OK;
    static bool configured = false;
    const int bytes = (int)sizeof(GradSmem);
    if (!configured) {
        if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
            return fail(BK_ERR_LAUNCH, "bk_mlp_gradient: cannot reserve shared memory");
        configured = true;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_mlp_grad<<<(unsigned)((batch + kRows - 1) / kRows), kRows, bytes, s>>>(batch, features, targets, to_norm(*norm),
                                                                            params, grads, loss_sum);
    return check_launch("bk_mlp_gradient");
}

int bk_mlp_adam(const float* grads, float* params, float* first_moment, float* second_moment, int32_t step,
                float learning_rate, float beta1, float beta2, float epsilon, void* stream) {
    if (!grads || !params || !first_moment || !second_moment || step < 1)
        return fail(BK_ERR_ARGUMENT, "bk_mlp_adam: bad argument");
    float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_mlp_adam<<<(kParamCount + 255) / 256, 256, 0, s>>>(kParamCount, params, grads, first_moment, second_moment,
                                                         learning_rate, beta1, beta2, epsilon, c1, c2);
    return check_launch("bk_mlp_adam");
}

int bk_mlp_pack(const float* params, void* packed, void* stream) {
    if (!params || !packed) return fail(BK_ERR_ARGUMENT, "bk_mlp_pack: null argument");
    if (reinterpret_cast<uintptr_t>(packed) % 16 != 0) return fail(BK_ERR_ARGUMENT, "bk_mlp_pack: packed weights must be 16-byte aligned");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_mlp_pack<<<(kHidden * kHidden + 255) / 256, 256, 0, s>>>(params, static_cast<unsigned char*>(packed));
    return check_launch("bk_mlp_pack");
}

}  // extern "C"
