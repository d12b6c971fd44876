// Internal helpers shared by the libbbpd translation units (not part of the ABI).
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "bbpd.h"

namespace bbpd {

// Record a message for bbpd_last_error() on this thread and return `code`.
int fail(int code, const char *fmt, ...);
void clear_error();

}  // namespace bbpd

#ifdef __CUDACC__
#include <cuda_runtime.h>

#define BBPD_CUDA_TRY(expr)                                                        \
    do {                                                                           \
        cudaError_t e_ = (expr);                                                   \
        if (e_ != cudaSuccess)                                                     \
            return bbpd::fail(e_ == cudaErrorMemoryAllocation ? BBPD_ERR_OOM      \
                                                              : BBPD_ERR_CUDA,    \
                              "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),     \
                              __FILE__, __LINE__);                                 \
    } while (0)

namespace bbpd {
// Fails with BBPD_ERR_NO_DEVICE when no CUDA device is visible: this library
// has no CPU implementation to fall back to.
int require_device();
inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
}  // namespace bbpd
#endif
