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

static std::atomic<int> g_bounds{-1};  // -1: not yet read from the environment

bool bounds_check_on() {
    int v = g_bounds.load();
    if (v < 0) {
        const char* e = getenv("MM_BOUNDS_CHECK");
        int want = (e && *e && *e != '0') ? 1 : 0, expect = -1;
        g_bounds.compare_exchange_strong(expect, want);
        v = g_bounds.load();
    }
    return v == 1;
}

void set_bounds_check(int on) { g_bounds.store(on ? 1 : 0); }

// cuMemGetAddressRange (driver API, resolved at run time: the library links
// only the runtime): base and size of the allocation that holds a pointer.
typedef int (*AddressRangeFn)(unsigned long long* base, size_t* size, unsigned long long ptr);

static AddressRangeFn address_range() {
    static std::atomic<int> state{0};  // 0 unresolved, 1 resolved, 2 unavailable
    static AddressRangeFn fn = nullptr;
    if (state.load() == 0) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess && f) {
            fn = reinterpret_cast<AddressRangeFn>(f);
            state.store(1);
        } else {
            cudaGetLastError();
            state.store(2);
        }
    }
    return state.load() == 1 ? fn : nullptr;
}

static int check_range_now(const void* p, size_t bytes, const char* who, const char* what) {
    if (bytes == 0) return MM_OK;
    if (p == nullptr) {
        set_error("%s: %s is NULL", who, what);
        return MM_EINVAL;
    }
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        set_error("%s: %s (%p) is not memory CUDA knows", who, what, p);
        return MM_EINVAL;
    }
    if (a.type == cudaMemoryTypeUnregistered) {
        set_error("%s: %s (%p) is pageable host memory; pass device memory", who, what, p);
        return MM_EINVAL;
    }
    int dev = 0;
    MM_CUDA(cudaGetDevice(&dev));
    if (a.type == cudaMemoryTypeDevice && a.device != dev) {
        set_error("%s: %s lives on device %d, the call runs on device %d", who, what, a.device, dev);
        return MM_EINVAL;
    }
    if (a.type == cudaMemoryTypeHost) return MM_OK;  // mapped pinned host memory: no range query
    AddressRangeFn fn = address_range();
    unsigned long long base = 0;
    size_t size = 0;
    if (fn && fn(&base, &size, (unsigned long long)(uintptr_t)p) == 0) {
        const unsigned long long off = (unsigned long long)(uintptr_t)p - base;
        if (off + bytes > size) {
            set_error("%s: %s needs %zu bytes but only %llu remain in its allocation (%zu bytes at offset %llu)",
                      who, what, bytes, (unsigned long long)(size - off), size, off);
            return MM_EINVAL;
        }
    }
    return MM_OK;
}

int check_range(const void* p, size_t bytes, const char* who, const char* what) {
    return bounds_check_on() ? check_range_now(p, bytes, who, what) : MM_OK;
}

}  // namespace mm

extern "C" int mm_check_array(const void* p, size_t bytes) {
    return mm::check_range_now(p, bytes, "mm_check_array", "array");
}

extern "C" int mm_version(void) { return 1; }

extern "C" int mm_set_bounds_check(int on) {
    mm::set_bounds_check(on);
    return MM_OK;
}

extern "C" int mm_get_bounds_check(void) { return mm::bounds_check_on() ? 1 : 0; }

extern "C" int mm_last_error(char* buf, size_t len) {
    size_t L = strlen(mm::g_err);
    if (buf && len) {
        size_t c = L < len - 1 ? L : len - 1;
        memcpy(buf, mm::g_err, c);
        buf[c] = 0;
    }
    return (int)L;
}
