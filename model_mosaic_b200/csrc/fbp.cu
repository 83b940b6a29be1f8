// FBP filter of processing/fbp_filter.py (vendored tomocupy FBPFilter) for sm_100a.
//
// Per sinogram row of n samples (processing/fbp_filter.py:128-192): replicate
// the edge samples to ne = 4n (pad = (ne - n)/2 on both sides), rfft, multiply
// by the real weights w[0..ne/2], irfft (divides by ne), keep the centre n.
// The weights are real and extend evenly over the full spectrum
// (W[k] = W[ne - k]), so the filter maps real rows to real rows and two rows
// packed as the real and imaginary parts of one complex line are filtered
// independently: one Stockham convolution of length ne (fft_smem.cuh) per two
// rows, in place, loads and stores straight from and to the rows.  Sizes
// outside the native range (ne not a power of two in [16, 8192]) run cuFFT
// R2C/C2R over chunks of rows through a scratch buffer.
#include "mm_common.cuh"
#include "fft_smem.cuh"

#include <math.h>

#include <algorithm>
#include <vector>

using mm::dev_alloc;

struct mm_fbp {
    int n = 0, ne = 0, chunk = 0;
    bool native = false;
    float2* tw = nullptr;       // native: Stockham twiddles, forward at 0, reversed at 2*ne
    float* pad = nullptr;       // general: (chunk, ne) padded rows
    float2* spec = nullptr;     // general: (chunk, ne/2 + 1) spectra
    cufftHandle r2c = 0, c2r = 0;
    int plan_rows = 0;
    size_t ws_bytes = 0;
};

namespace {

// Two rows per block: r0 = 2*blockIdx.x in the real part, r0 + 1 in the
// imaginary part (zero when absent).  Powers of two: bounded to 64 registers
// so that 1024 threads share an SM (two 8192-point lines), faster than one
// block at 128 registers despite a few spills; 3 * 2^k lengths (24 values
// per thread) at 128 registers.
template <int L>
__global__ void __launch_bounds__(stockham::Sched<L>::G,
                                  stockham::Sched<L>::P2
                                      ? (stockham::Sched<L>::G >= 32 ? 1024 / stockham::Sched<L>::G : 32)
                                      : 512 / (stockham::Sched<L>::G >= 32 ? stockham::Sched<L>::G : 32))
    k_fbp_filter(float* __restrict__ rows, long nrows,
                                                                      const float* __restrict__ w,
                                                                      const float2* __restrict__ tw, int n,
                                                                      float inv_ne) {
    extern __shared__ float2 sm[];
    const int g = threadIdx.x;
    const long r0 = 2L * blockIdx.x;
    const bool has1 = r0 + 1 < nrows;
    float* a = rows + r0 * n;
    float* b = a + n;
    const int pad = (L - n) / 2;
    const stockham::RowAddr ad{0};
    auto ld = [&](int pos) -> float2 {  // edge-replicated padding
        int i = pos - pad;
        i = i < 0 ? 0 : (i >= n ? n - 1 : i);
        return make_float2(a[i], has1 ? b[i] : 0.f);
    };
    auto mul = [&](int k, float2 v) -> float2 {
        const float wk = __ldg(w + (k <= L / 2 ? k : L - k)) * inv_ne;
        return make_float2(v.x * wk, v.y * wk);
    };
    auto st = [&](int pos, float2 v) {  // crop: every row is read before any is written
        const int i = pos - pad;
        if (i >= 0 && i < n) {
            a[i] = v.x;
            if (has1) b[i] = v.y;
        }
    };
    stockham::conv<L>(sm, ad, ld, mul, st, g, tw, tw + 2 * L);
}

template <int L>
int launch_native(mm_fbp* h, float* rows, long nrows, const float* w, cudaStream_t st) {
    const size_t smem = (size_t)(L + L / 16) * sizeof(float2);
    auto kern = k_fbp_filter<L>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long blocks = (nrows + 1) / 2;
    kern<<<(unsigned)blocks, stockham::Sched<L>::G, smem, st>>>(rows, nrows, w, h->tw, h->n, 1.0f / (float)L);
    MM_LAUNCHED();
    return MM_OK;
}

int dispatch_native(mm_fbp* h, float* rows, long nrows, const float* w, cudaStream_t st) {
    switch (h->ne) {
        case 16: return launch_native<16>(h, rows, nrows, w, st);
        case 32: return launch_native<32>(h, rows, nrows, w, st);
        case 64: return launch_native<64>(h, rows, nrows, w, st);
        case 128: return launch_native<128>(h, rows, nrows, w, st);
        case 256: return launch_native<256>(h, rows, nrows, w, st);
        case 512: return launch_native<512>(h, rows, nrows, w, st);
        case 1024: return launch_native<1024>(h, rows, nrows, w, st);
        case 2048: return launch_native<2048>(h, rows, nrows, w, st);
        case 4096: return launch_native<4096>(h, rows, nrows, w, st);
        case 8192: return launch_native<8192>(h, rows, nrows, w, st);
        case 96: return launch_native<96>(h, rows, nrows, w, st);
        case 192: return launch_native<192>(h, rows, nrows, w, st);
        case 384: return launch_native<384>(h, rows, nrows, w, st);
        case 768: return launch_native<768>(h, rows, nrows, w, st);
        case 1536: return launch_native<1536>(h, rows, nrows, w, st);
        case 3072: return launch_native<3072>(h, rows, nrows, w, st);
        case 6144: return launch_native<6144>(h, rows, nrows, w, st);
        case 12288: return launch_native<12288>(h, rows, nrows, w, st);
    }
    MM_REQUIRE(false, "FBP filter: no native kernel for ne=%d", h->ne);
}

// General sizes: edge-pad into scratch, multiply the spectrum, crop back.
__global__ void k_fbp_pad(const float* __restrict__ rows, float* __restrict__ pad, int n, int ne, long total) {
    const int p0 = (ne - n) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long r = i / ne;
        int c = (int)(i % ne) - p0;
        c = c < 0 ? 0 : (c >= n ? n - 1 : c);
        pad[i] = rows[r * n + c];
    }
}

__global__ void k_fbp_mul(float2* __restrict__ spec, const float* __restrict__ w, int nh, long total, float inv_ne) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const float wk = __ldg(w + i % nh) * inv_ne;
        spec[i] = make_float2(spec[i].x * wk, spec[i].y * wk);
    }
}

__global__ void k_fbp_crop(const float* __restrict__ pad, float* __restrict__ rows, int n, int ne, long total) {
    const int p0 = (ne - n) / 2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const long r = i / n;
        rows[i] = pad[r * ne + p0 + (int)(i % n)];
    }
}

int general_plans(mm_fbp* h, int rows) {
    if (h->plan_rows == rows) return MM_OK;
    if (h->r2c) cufftDestroy(h->r2c);
    if (h->c2r) cufftDestroy(h->c2r);
    h->r2c = h->c2r = 0;
    h->plan_rows = 0;
    int len[1] = {h->ne};
    const int nh = h->ne / 2 + 1;
    MM_CUFFT(cufftPlanMany(&h->r2c, 1, len, nullptr, 1, h->ne, nullptr, 1, nh, CUFFT_R2C, rows));
    MM_CUFFT(cufftPlanMany(&h->c2r, 1, len, nullptr, 1, nh, nullptr, 1, h->ne, CUFFT_C2R, rows));
    h->plan_rows = rows;
    return MM_OK;
}

int run_general(mm_fbp* h, float* rows, long nrows, const float* w, cudaStream_t st) {
    const int n = h->n, ne = h->ne, nh = ne / 2 + 1;
    const int bs = 256;
    for (long r0 = 0; r0 < nrows; r0 += h->chunk) {
        const int nr = (int)std::min<long>(h->chunk, nrows - r0);
        MM_TRY(general_plans(h, nr));
        const long tp = (long)nr * ne, tq = (long)nr * nh, tr = (long)nr * n;
        auto grid = [&](long t) { return (unsigned)std::min<long>((t + bs - 1) / bs, 148L * 32); };
        k_fbp_pad<<<grid(tp), bs, 0, st>>>(rows + r0 * n, h->pad, n, ne, tp);
        MM_LAUNCHED();
        MM_CUFFT(cufftSetStream(h->r2c, st));
        MM_CUFFT(cufftExecR2C(h->r2c, h->pad, (cufftComplex*)h->spec));
        k_fbp_mul<<<grid(tq), bs, 0, st>>>(h->spec, w, nh, tq, 1.0f / (float)ne);
        MM_LAUNCHED();
        MM_CUFFT(cufftSetStream(h->c2r, st));
        MM_CUFFT(cufftExecC2R(h->c2r, (cufftComplex*)h->spec, h->pad));
        k_fbp_crop<<<grid(tr), bs, 0, st>>>(h->pad, rows + r0 * n, n, ne, tr);
        MM_LAUNCHED();
    }
    return MM_OK;
}

void destroy(mm_fbp* h) {
    if (h->r2c) cufftDestroy(h->r2c);
    if (h->c2r) cufftDestroy(h->c2r);
    void* bufs[] = {h->tw, h->pad, h->spec};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete h;
}

}  // namespace

extern "C" int mm_fbp_create(int n, int batch_chunk, mm_fbp** out) {
    MM_REQUIRE(out != nullptr, "mm_fbp_create: out is NULL");
    *out = nullptr;
    MM_REQUIRE(n >= 2 && n <= (1 << 20), "mm_fbp_create: n=%d out of range", n);
    MM_REQUIRE(batch_chunk >= 1, "mm_fbp_create: batch_chunk must be positive");
    MM_CUDA(mmfft::init_constants());
    mm_fbp* h = new mm_fbp();
    h->n = n;
    h->ne = 4 * n;
    h->chunk = batch_chunk;
    // native padded lengths: powers of two in [16, 8192], 3 * 2^k in [96, 12288]
    h->native = mm_is_pow2(h->ne) ? (h->ne >= 16 && h->ne <= 8192)
                                  : (stockham::length_ok(h->ne) && h->ne >= 96 && h->ne <= 12288);
    int rc = MM_OK;
    if (h->native) {
        std::vector<float2> tw(4 * (size_t)h->ne, make_float2(0.f, 0.f));
        stockham::host_twiddles(h->ne, false, tw.data());
        stockham::host_twiddles(h->ne, true, tw.data() + 2 * (size_t)h->ne);
        rc = dev_alloc((void**)&h->tw, tw.size() * sizeof(float2), "FBP twiddles");
        if (rc == MM_OK &&
            cudaMemcpy(h->tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
            mm::set_error("mm_fbp_create: table upload failed");
            rc = MM_ECUDA;
        }
        h->ws_bytes = tw.size() * sizeof(float2);
    } else {
        rc = dev_alloc((void**)&h->pad, (size_t)batch_chunk * h->ne * sizeof(float), "FBP padded rows");
        if (rc == MM_OK)
            rc = dev_alloc((void**)&h->spec, (size_t)batch_chunk * (h->ne / 2 + 1) * sizeof(float2), "FBP spectra");
        h->ws_bytes = (size_t)batch_chunk * h->ne * 4 + (size_t)batch_chunk * (h->ne / 2 + 1) * 8;
    }
    if (rc != MM_OK) {
        destroy(h);
        return rc;
    }
    *out = h;
    return MM_OK;
}

extern "C" int mm_fbp_destroy(mm_fbp* h) {
    if (!h) return MM_OK;
    cudaDeviceSynchronize();
    destroy(h);
    return MM_OK;
}

extern "C" int mm_fbp_filter(mm_fbp* h, float* sino, long rows, const float* w, void* stream) {
    MM_REQUIRE(h != nullptr, "mm_fbp_filter: NULL handle");
    MM_REQUIRE(sino != nullptr && w != nullptr, "mm_fbp_filter: NULL array");
    MM_REQUIRE(rows >= 0, "mm_fbp_filter: rows=%ld negative", rows);
    MM_REQUIRE(((uintptr_t)sino % 4) == 0 && ((uintptr_t)w % 4) == 0, "mm_fbp_filter: misaligned array");
    if (rows == 0) return MM_OK;
    MM_RANGE(sino, (size_t)rows * h->n * 4, "mm_fbp_filter", "sino");
    MM_RANGE(w, (size_t)(h->ne / 2 + 1) * 4, "mm_fbp_filter", "w");
    cudaStream_t st = (cudaStream_t)stream;
    return h->native ? dispatch_native(h, sino, rows, w, st) : run_general(h, sino, rows, w, st);
}

extern "C" size_t mm_fbp_workspace_bytes(const mm_fbp* h) { return h ? h->ws_bytes : 0; }
