// Optional per-kernel CUDA-event timing inside the fused entry points (off unless bk_profile_start ran).
#pragma once
#include <cuda_runtime.h>

namespace bk {
// Record an event pair around the next launch named `name` on `stream` (no-op when profiling is off).
int profile_begin(const char* name, cudaStream_t stream);
void profile_end(int record, cudaStream_t stream);
}  // namespace bk
