// Shared helpers of the model_mosaic_b200 CUDA library: status codes, the
// per-thread last-error text and checked wrappers around CUDA/cuFFT calls.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/mosaic.h"

#include <vector>

namespace mm {

// Optional per-stage CUDA-event timing of a handle's launches (off by
// default).  begin()/end() bracket one stage on the caller's stream; read()
// waits for the recorded events and adds their elapsed times per stage.
struct StageTimer {
    static constexpr int kMax = 16;
    bool on = false;
    double ms[kMax] = {0};
    long long calls[kMax] = {0};
    long long kernels = 0;  // launches of this library's own kernels while on
    struct Rec { int stage; cudaEvent_t a, b; };
    std::vector<Rec> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t cur_a = nullptr;
    int cur_stage = -1;

    cudaEvent_t take() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(int stage, cudaStream_t st) {
        if (!on) return;
        cur_stage = stage;
        cur_a = take();
        cudaEventRecord(cur_a, st);
    }
    void end(cudaStream_t st, int own_kernels) {
        if (!on || cur_stage < 0) return;
        cudaEvent_t b = take();
        cudaEventRecord(b, st);
        pending.push_back({cur_stage, cur_a, b});
        kernels += own_kernels;
        cur_stage = -1;
        if (pending.size() > 4096) read();  // bound the event backlog
    }
    void read() {
        for (auto& r : pending) {
            float t = 0.f;
            cudaEventSynchronize(r.b);
            cudaEventElapsedTime(&t, r.a, r.b);
            ms[r.stage] += t;
            calls[r.stage] += 1;
            pool.push_back(r.a);
            pool.push_back(r.b);
        }
        pending.clear();
    }
    void reset() {
        read();
        for (int i = 0; i < kMax; ++i) { ms[i] = 0; calls[i] = 0; }
        kernels = 0;
    }
    void release() {
        read();
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
        pool.clear();
    }
};

void set_error(const char* fmt, ...);
const char* cufft_name(cufftResult r);

// Allocation hook for fault-injection tests: when the environment variable
// MM_FAIL_ALLOC_AFTER=k is set, the (k+1)-th device allocation made through
// dev_alloc() in this process reports MM_ENOMEM without calling cudaMalloc.
int dev_alloc(void** p, size_t bytes, const char* what);

// Caller-array checks (off by default; mm_set_bounds_check(1) or the
// environment variable MM_BOUNDS_CHECK=1 turn them on).  When on, every
// compute entry point checks each array it is given before it launches
// anything: [p, p + bytes) must be device memory of the current device (or
// mapped pinned host memory) and lie inside one allocation.  A failed check
// returns MM_EINVAL and names the argument, so a short buffer is reported
// instead of being written past.  Sub-allocators that carve arrays out of
// larger cudaMalloc blocks (torch's caching allocator) are checked against
// the block.
bool bounds_check_on();
int check_range(const void* p, size_t bytes, const char* who, const char* what);

}  // namespace mm

#define MM_RANGE(p, bytes, who, what) MM_TRY(mm::check_range((p), (bytes), (who), (what)))

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
