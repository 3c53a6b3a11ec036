// Error reporting shared by the C-ABI translation units (one thread-local message buffer).
#pragma once

namespace bk {
// Record `msg` as the calling thread's last error and return `code`.
int fail(int code, const char* msg);
// Turn a pending CUDA launch error into BK_ERR_LAUNCH with a message naming `name`.
int check_launch(const char* name);
}  // namespace bk
