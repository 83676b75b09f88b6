// Error reporting shared by every translation unit of libxpbd_b200.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/xpbd_b200.h"

namespace xpbd {

// Dynamic shared memory above this asks for the opt-in attribute.  The default
// per-block limit (48 KB) counts static shared memory too, so opting in only
// above 48 KB of dynamic memory would leave kernels with a little static
// memory unlaunchable just below it.
constexpr size_t kSmemOptIn = 40 * 1024;

// Last error of the calling host thread (returned by xpbd_error_string()).
char* err_buffer();

inline int fail(int code, const char* msg) {
    snprintf(err_buffer(), 256, "%s", msg);
    return code;
}
inline int cuda_check(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(err_buffer(), 256, "%s: %s", where, cudaGetErrorString(e));
        return XPBD_ERR_CUDA;
    }
    return XPBD_OK;
}
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace xpbd
