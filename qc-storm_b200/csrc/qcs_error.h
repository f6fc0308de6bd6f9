// Error reporting shared by the C-ABI translation units: a status code is
// returned, the message is kept per thread for qcs_last_error().
#pragma once

#include <cuda_runtime.h>

namespace qcs {

// Records `what` (plus the CUDA error text when e is set) and returns code.
int fail(int code, const char *what, cudaError_t e = cudaSuccess);

}  // namespace qcs

#define QCS_CUDA(call, what)                                             \
    do {                                                                 \
        cudaError_t e_ = (call);                                         \
        if (e_ != cudaSuccess) return qcs::fail(QCS_ERR_CUDA, what, e_); \
    } while (0)
