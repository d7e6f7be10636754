// Internal helpers shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

namespace ctc {
int fail(int status, const char *fmt, ...);   // records the message, returns status
int *dev_err_ptr();                           // device failure word of the current device
}  // namespace ctc

#define CUDA_TRY(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return ctc::fail(CTC_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
    } while (0)
