// Status text, allocation hook and library version for the C-ABI.
#include "mm_common.cuh"

#include <stdlib.h>
#include <string.h>

#include <atomic>

namespace mm {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char* cufft_name(cufftResult r) {
    switch (r) {
        case CUFFT_SUCCESS: return "CUFFT_SUCCESS";
        case CUFFT_INVALID_PLAN: return "CUFFT_INVALID_PLAN";
        case CUFFT_ALLOC_FAILED: return "CUFFT_ALLOC_FAILED";
        case CUFFT_INVALID_TYPE: return "CUFFT_INVALID_TYPE";
        case CUFFT_INVALID_VALUE: return "CUFFT_INVALID_VALUE";
        case CUFFT_INTERNAL_ERROR: return "CUFFT_INTERNAL_ERROR";
        case CUFFT_EXEC_FAILED: return "CUFFT_EXEC_FAILED";
        case CUFFT_SETUP_FAILED: return "CUFFT_SETUP_FAILED";
        case CUFFT_INVALID_SIZE: return "CUFFT_INVALID_SIZE";
        case CUFFT_INCOMPLETE_PARAMETER_LIST: return "CUFFT_INCOMPLETE_PARAMETER_LIST";
        case CUFFT_INVALID_DEVICE: return "CUFFT_INVALID_DEVICE";
        case CUFFT_NO_WORKSPACE: return "CUFFT_NO_WORKSPACE";
        case CUFFT_NOT_IMPLEMENTED: return "CUFFT_NOT_IMPLEMENTED";
        case CUFFT_NOT_SUPPORTED: return "CUFFT_NOT_SUPPORTED";
        default: return "cuFFT error";
    }
}

static std::atomic<long> g_alloc_count{0};

int dev_alloc(void** p, size_t bytes, const char* what) {
    *p = nullptr;
    const char* lim = getenv("MM_FAIL_ALLOC_AFTER");
    if (lim && *lim) {
        long k = atol(lim);
        if (g_alloc_count.fetch_add(1) >= k) {
            set_error("injected allocation failure (MM_FAIL_ALLOC_AFTER=%ld) for %s", k, what);
            return MM_ENOMEM;
        }
    }
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error("cudaMalloc(%zu bytes) for %s failed: %s", bytes, what, cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? MM_ENOMEM : MM_ECUDA;
    }
    return MM_OK;
}

}  // namespace mm

extern "C" int mm_version(void) { return 1; }

extern "C" int mm_last_error(char* buf, size_t len) {
    size_t L = strlen(mm::g_err);
    if (buf && len) {
        size_t c = L < len - 1 ? L : len - 1;
        memcpy(buf, mm::g_err, c);
        buf[c] = 0;
    }
    return (int)L;
}
