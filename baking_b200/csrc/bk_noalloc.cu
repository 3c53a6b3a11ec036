// A mechanics substep that needs no device memory from the caller beyond its particle arrays.
//
// bk_substep takes its background grid (momentum/mass and velocity nodes plus the active-box
// bounds) from the caller, who allocates it with cudaMalloc or a framework allocator. Some
// callers cannot do that: code running where the device allocator must not be touched (inside
// an allocator hook, a signal-safe or real-time path, or a host that forbids runtime
// allocation after start-up) still needs to advance a small simulation. bk_substep_static_grid
// serves them: its grid lives in a fixed array compiled into this library, so the call
// allocates and frees nothing.
//
// Limits and sharing. The array holds at most kMaxNodes grid nodes (48^3, about 3.4 MB) and is
// resident on every GPU that loads this library until the process exits. It is shared by every
// call on a device and keeps the last call's contents, so each call first resets the part it uses;
// calls whose executions overlap on the GPU (different streams or threads) race on it and must
// be serialised by the caller.
//
// Start-up. Under lazy module loading (CUDA_MODULE_LOADING=LAZY, the default since CUDA 12.2) the
// module holding the array is loaded, and the array's device memory reserved, by the first call
// in each CUDA context. That first call may therefore allocate; a caller that must not allocate
// later makes one call per device (and per context it uses) at start-up, before any stream
// capture. Every call works in whatever context is current: primary or not, before or after a
// cudaDeviceReset.
#include <climits>
#include <cstdio>

#include "baking_b200.h"
#include "bk_common.h"

namespace {

constexpr int kMaxResolution = 48;
constexpr long long kMaxNodes = (long long)kMaxResolution * kMaxResolution * kMaxResolution;
constexpr long long kNodeBytes = 16;                              // one float4 per node and field
constexpr long long kBoundsOffset = 2 * kMaxNodes * kNodeBytes;  // after node_pm and node_v
constexpr long long kScratchBytes = kBoundsOffset + 256;

// The grid scratch of bk_substep_static_grid: node_pm, then node_v, then 12 ints of bounds.
static __device__ __align__(256) unsigned char g_grid_scratch[kScratchBytes];

// Device address of g_grid_scratch in the current context. The host symbol g_grid_scratch is only
// a handle: its host address must never reach a kernel. The address is looked up on every call
// rather than cached per device: after cudaDeviceReset, or with a non-primary context made current
// (cuCtxCreate/cuCtxSetCurrent), the array lives at another address, and once the module is
// loaded in the context the lookup allocates nothing.
int scratch_address(void** out) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_grid_scratch);
    if (e != cudaSuccess || !ptr) {
        char msg[256];
        snprintf(msg, sizeof msg, "bk_substep_static_grid: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return bk::fail(BK_ERR_LAUNCH, msg);
    }
    *out = ptr;
    return BK_OK;
}

// Zero the nodes of a resolution^3 grid and mark both active boxes empty, the state bk_substep
// expects of a fresh grid.
__global__ void k_reset_static_grid(float4* pm, float4* v, int* bounds, long long nodes) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < 12 && bounds) {
        int k = (int)(i % 6);
        bounds[i] = k < 3 ? INT_MAX : INT_MIN;
    }
    for (; i < nodes; i += (long long)gridDim.x * blockDim.x) {
        pm[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        v[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

}  // namespace

extern "C" {

int bk_substep_static_grid(const BkSubstepParams* params, const BkState* in, BkState* out,
                           const BkConstants* constants, BkDiagnostics* diagnostics, BkFlags* flags, void* stream) {
    if (!params || !in || !out || !constants || !diagnostics || !flags)
        return bk::fail(BK_ERR_ARGUMENT, "bk_substep_static_grid: null argument");
    if (params->transport || params->gas)
        return bk::fail(BK_ERR_UNSUPPORTED,
                        "bk_substep_static_grid: the static grid holds mechanics nodes only; transport/gas need bk_substep");
    if (params->resolution < 4 || params->resolution > kMaxResolution) {
        char msg[160];
        snprintf(msg, sizeof msg, "bk_substep_static_grid: grid resolution %d is outside 4..%d (the static grid holds %lld nodes)",
                 params->resolution, kMaxResolution, kMaxNodes);
        return bk::fail(BK_ERR_ARGUMENT, msg);
    }
    void* base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    unsigned char* bytes = static_cast<unsigned char*>(base);
    const long long nodes = (long long)params->resolution * params->resolution * params->resolution;
    float4* pm = reinterpret_cast<float4*>(bytes);
    float4* v = reinterpret_cast<float4*>(bytes + kMaxNodes * kNodeBytes);
    int* bounds = reinterpret_cast<int*>(bytes + kBoundsOffset);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    k_reset_static_grid<<<(unsigned)((nodes + 255) / 256), 256, 0, s>>>(pm, v, bounds, nodes);
    if (int rc = bk::check_launch("bk_substep_static_grid/reset")) return rc;
    BkGrid grid = {};
    grid.node_pm = reinterpret_cast<float*>(pm);
    grid.node_v = reinterpret_cast<float*>(v);
    grid.bounds = bounds;
    return bk_substep(params, in, out, constants, &grid, nullptr, diagnostics, flags, BK_PHASE_MECHANICS, stream);
}

}  // extern "C"
