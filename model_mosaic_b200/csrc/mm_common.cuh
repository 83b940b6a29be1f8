// Shared helpers of the model_mosaic_b200 CUDA library: status codes, the
// per-thread last-error text and checked wrappers around CUDA/cuFFT calls.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/mosaic.h"

namespace mm {

void set_error(const char* fmt, ...);
const char* cufft_name(cufftResult r);

// Allocation hook for fault-injection tests: when the environment variable
// MM_FAIL_ALLOC_AFTER=k is set, the (k+1)-th device allocation made through
// dev_alloc() in this process reports MM_ENOMEM without calling cudaMalloc.
int dev_alloc(void** p, size_t bytes, const char* what);

}  // namespace mm

#define MM_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            mm::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,               \
                          cudaGetErrorString(e_));                                 \
            return MM_ECUDA;                                                       \
        }                                                                          \
    } while (0)

#define MM_CUFFT(call)                                                             \
    do {                                                                           \
        cufftResult r_ = (call);                                                   \
        if (r_ != CUFFT_SUCCESS) {                                                 \
            mm::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,               \
                          mm::cufft_name(r_));                                     \
            return MM_ECUFFT;                                                      \
        }                                                                          \
    } while (0)

#define MM_TRY(expr)                                                               \
    do {                                                                           \
        int s_ = (expr);                                                           \
        if (s_ != MM_OK) return s_;                                                \
    } while (0)

#define MM_REQUIRE(cond, ...)                                                      \
    do {                                                                           \
        if (!(cond)) {                                                             \
            mm::set_error(__VA_ARGS__);                                            \
            return MM_EINVAL;                                                      \
        }                                                                          \
    } while (0)

// Kernel launches: check the launch itself (configuration errors) only; the
// kernels carry no device-side asserts.
#define MM_LAUNCHED() MM_CUDA(cudaGetLastError())

static __host__ __device__ inline int mm_is_pow2(long x) { return x > 0 && (x & (x - 1)) == 0; }
