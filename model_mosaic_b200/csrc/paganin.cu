// Paganin single-distance phase retrieval (processing/paganin.py) for sm_100a.
//
// Per (nz, n) intensity frame I (processing/paganin.py:64-91):
//   phase = -log(clip(irfft2(H * rfft2(I)), 1e-6)),
//   H(ky, kx) = alpha / (lambda z (kx^2 + ky^2) / (4 pi) + alpha)  (real, even).
// H is not separable, so the transform runs as three passes over HBM:
//   1. rows: two real rows packed as one complex line, FFT_n, unpacked into
//      their half spectra (k = 0 .. n/2) in `spec` (frames, nz, n/2+1);
//   2. columns of spec: FFT_nz, * H / (n nz), IFFT_nz, in place (one Stockham
//      convolution per column, fft_smem.cuh);
//   3. rows: two half spectra rebuilt into one Hermitian-paired complex line
//      in the load, IFFT_n, -log(max(., 1e-6)) of the real and imaginary parts
//      in the store.
// 24 bytes of HBM traffic per pixel (4 in, 8 + 8 through spec, 4 out).  Sizes
// outside the native range (n, nz powers of two in [2, 4096]) use cuFFT
// R2C/C2R over all frames, as the reference does.
#include "mm_common.cuh"
#include "fft_smem.cuh"

#include <math.h>

#include <algorithm>
#include <vector>

using mm::dev_alloc;

struct mm_pgn {
    int n = 0, nz = 0, ntheta = 0, nh = 0;
    bool native = false;
    float* H = nullptr;        // (nz, n/2 + 1)
    float2* spec = nullptr;    // (ntheta, nz, n/2 + 1)
    float2* twx = nullptr;     // native: n-point tables, forward at 0, reversed at 2n
    float2* twy = nullptr;     // native: nz-point tables, forward at 0, reversed at 2nz
    float* real = nullptr;     // general: (ntheta, nz, n)
    cufftHandle r2c = 0, c2r = 0;
    size_t ws_bytes = 0;
};

namespace {

template <int N>
constexpr int rows_per_block() {
    constexpr int G = stockham::Sched<N>::G;
    return G >= 256 ? 1 : 256 / G;
}
template <int N>
constexpr int cols_per_block() {
    constexpr int G = stockham::Sched<N>::G;
    return 256 / G < 4 ? 4 : (256 / G > 32 ? 32 : 256 / G);
}

// Pass 1: rows 2p (real part) and 2p+1 (imaginary part) -> half spectra.
template <int N, int RPB>
__global__ void __launch_bounds__(RPB * stockham::Sched<N>::G) k_pg_xfwd(const float* __restrict__ I,
                                                                         float2* __restrict__ spec, long rows,
                                                                         const float2* __restrict__ tw) {
    constexpr int G = stockham::Sched<N>::G, NH = N / 2 + 1, LP = N + N / 16;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x, rr = threadIdx.y;
    const long ra = 2 * ((long)blockIdx.x * RPB + rr), rb = ra + 1;
    const bool live = ra < rows, hasb = rb < rows;
    const stockham::RowAddr ad{rr * LP};
    auto ld = [&](int pos) -> float2 {
        return make_float2(live ? __ldg(I + ra * N + pos) : 0.f, hasb ? __ldg(I + rb * N + pos) : 0.f);
    };
    auto st = [&](int pos, float2 v) { sm[ad(pos)] = v; };
    stockham::fft<N, false>(sm, ad, ld, st, g, tw);
    __syncthreads();
    if (!live) return;
    for (int k = g; k < NH; k += G) {
        const float2 z1 = sm[ad(k)], z2 = sm[ad(k == 0 ? 0 : N - k)];
        // Za = (Z[k] + conj Z[N-k]) / 2, Zb = (Z[k] - conj Z[N-k]) / (2i)
        spec[ra * NH + k] = make_float2(0.5f * (z1.x + z2.x), 0.5f * (z1.y - z2.y));
        if (hasb) spec[rb * NH + k] = make_float2(0.5f * (z1.y + z2.y), -0.5f * (z1.x - z2.x));
    }
}

// Pass 2: column (frame t, bin k) of spec along z: FFT, * H[ky][k] * scale, IFFT.
template <int NZ, int CW>
__global__ void __launch_bounds__(CW * stockham::Sched<NZ>::G) k_pg_ycol(float2* __restrict__ spec,
                                                                         const float* __restrict__ H, int nh,
                                                                         const float2* __restrict__ tw,
                                                                         float scale) {
    extern __shared__ float2 sm[];
    const int c = threadIdx.x, g = threadIdx.y;
    const int col = blockIdx.x * CW + c;
    const bool live = col < nh;
    float2* frame = spec + (long)blockIdx.y * NZ * nh;
    const stockham::ColAddr<CW> ad{c};
    auto ld = [&](int pos) -> float2 { return live ? frame[(long)pos * nh + col] : make_float2(0.f, 0.f); };
    auto mul = [&](int ky, float2 v) -> float2 {
        const float h = live ? __ldg(H + (long)ky * nh + col) * scale : 0.f;
        return make_float2(v.x * h, v.y * h);
    };
    auto st = [&](int pos, float2 v) {
        if (live) frame[(long)pos * nh + col] = v;
    };
    stockham::conv<NZ>(sm, ad, ld, mul, st, g, tw, tw + 2 * NZ);
}

// Pass 3: half spectra of rows 2p, 2p+1 -> Z = Za + i Zb over the full line
// (Z[N-k] = conj Za[k] + i conj Zb[k]), IFFT, -log(max(., 1e-6)).
template <int N, int RPB>
__global__ void __launch_bounds__(RPB * stockham::Sched<N>::G) k_pg_xinv(const float2* __restrict__ spec,
                                                                         float* __restrict__ out, long rows,
                                                                         const float2* __restrict__ tw) {
    constexpr int NH = N / 2 + 1, LP = N + N / 16;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x, rr = threadIdx.y;
    const long ra = 2 * ((long)blockIdx.x * RPB + rr), rb = ra + 1;
    const bool live = ra < rows, hasb = rb < rows;
    const stockham::RowAddr ad{rr * LP};
    auto ld = [&](int pos) -> float2 {
        const bool lo = pos <= N / 2;
        const int k = lo ? pos : N - pos;
        const float2 a = live ? __ldg(spec + ra * NH + k) : make_float2(0.f, 0.f);
        const float2 b = hasb ? __ldg(spec + rb * NH + k) : make_float2(0.f, 0.f);
        return lo ? make_float2(a.x - b.y, a.y + b.x) : make_float2(a.x + b.y, b.x - a.y);
    };
    auto st = [&](int pos, float2 v) {
        if (live) out[ra * N + pos] = -logf(fmaxf(v.x, 1e-6f));
        if (hasb) out[rb * N + pos] = -logf(fmaxf(v.y, 1e-6f));
    };
    stockham::fft<N, true>(sm, ad, ld, st, g, tw);
}

template <int N>
int launch_rows(const mm_pgn* h, bool inverse, const float* I, float* out, long rows, cudaStream_t st) {
    constexpr int G = stockham::Sched<N>::G, RPB = rows_per_block<N>();
    const size_t smem = (size_t)RPB * (N + N / 16) * sizeof(float2);
    const long pairs = (rows + 1) / 2;
    dim3 block(G, RPB), grid((unsigned)((pairs + RPB - 1) / RPB));
    if (!inverse) {
        auto kern = k_pg_xfwd<N, RPB>;
        MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, block, smem, st>>>(I, h->spec, rows, h->twx);
    } else {
        auto kern = k_pg_xinv<N, RPB>;
        MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, block, smem, st>>>(h->spec, out, rows, h->twx);
    }
    MM_LAUNCHED();
    return MM_OK;
}

template <int NZ>
int launch_cols(const mm_pgn* h, int frames, cudaStream_t st) {
    constexpr int G = stockham::Sched<NZ>::G, CW = cols_per_block<NZ>();
    const size_t smem = (size_t)stockham::ColAddr<CW>::rows(NZ) * CW * sizeof(float2);
    auto kern = k_pg_ycol<NZ, CW>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 block(CW, G), grid((unsigned)((h->nh + CW - 1) / CW), (unsigned)frames);
    kern<<<grid, block, smem, st>>>(h->spec, h->H, h->nh, h->twy, 1.0f / ((float)h->n * (float)h->nz));
    MM_LAUNCHED();
    return MM_OK;
}

#define MM_LINE_SWITCH(x, F, ...)                                              \
    switch (x) {                                                               \
        case 2: return F<2>(__VA_ARGS__);                                      \
        case 4: return F<4>(__VA_ARGS__);                                      \
        case 8: return F<8>(__VA_ARGS__);                                      \
        case 16: return F<16>(__VA_ARGS__);                                    \
        case 32: return F<32>(__VA_ARGS__);                                    \
        case 64: return F<64>(__VA_ARGS__);                                    \
        case 128: return F<128>(__VA_ARGS__);                                  \
        case 256: return F<256>(__VA_ARGS__);                                  \
        case 512: return F<512>(__VA_ARGS__);                                  \
        case 1024: return F<1024>(__VA_ARGS__);                                \
        case 2048: return F<2048>(__VA_ARGS__);                                \
        case 4096: return F<4096>(__VA_ARGS__);                                \
        case 96: return F<96>(__VA_ARGS__);                                    \
        case 192: return F<192>(__VA_ARGS__);                                  \
        case 384: return F<384>(__VA_ARGS__);                                  \
        case 768: return F<768>(__VA_ARGS__);                                  \
        case 1536: return F<1536>(__VA_ARGS__);                                \
        case 3072: return F<3072>(__VA_ARGS__);                                \
    }

int rows_pass(const mm_pgn* h, bool inverse, const float* I, float* out, long rows, cudaStream_t st) {
    MM_LINE_SWITCH(h->n, launch_rows, h, inverse, I, out, rows, st)
    MM_REQUIRE(false, "Paganin: no native row kernel for n=%d", h->n);
}

int cols_pass(const mm_pgn* h, int frames, cudaStream_t st) {
    MM_LINE_SWITCH(h->nz, launch_cols, h, frames, st)
    MM_REQUIRE(false, "Paganin: no native column kernel for nz=%d", h->nz);
}
#undef MM_LINE_SWITCH

// General sizes: the reference's rfft2 * H -> irfft2 over all ntheta frames
// (tail frames zeroed), then -log(clip).
__global__ void k_pg_mul(float2* __restrict__ spec, const float* __restrict__ H, long per_frame, long total,
                         float scale) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const float h = __ldg(H + i % per_frame) * scale;
        spec[i] = make_float2(spec[i].x * h, spec[i].y * h);
    }
}

__global__ void k_pg_log(const float* __restrict__ x, float* __restrict__ out, long total) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x)
        out[i] = -logf(fmaxf(x[i], 1e-6f));
}

unsigned grid_of(long total) { return (unsigned)std::min<long>((total + 255) / 256, 148L * 32); }

int run_general(mm_pgn* h, const float* I, float* out, int frames, cudaStream_t st) {
    const long fr = (long)h->nz * h->n, fs = (long)h->nz * h->nh;
    MM_CUDA(cudaMemcpyAsync(h->real, I, frames * fr * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (frames < h->ntheta)
        MM_CUDA(cudaMemsetAsync(h->real + frames * fr, 0, (h->ntheta - frames) * fr * sizeof(float), st));
    MM_CUFFT(cufftSetStream(h->r2c, st));
    MM_CUFFT(cufftExecR2C(h->r2c, h->real, (cufftComplex*)h->spec));
    k_pg_mul<<<grid_of(h->ntheta * fs), 256, 0, st>>>(h->spec, h->H, fs, h->ntheta * fs,
                                                      1.0f / ((float)h->n * (float)h->nz));
    MM_LAUNCHED();
    MM_CUFFT(cufftSetStream(h->c2r, st));
    MM_CUFFT(cufftExecC2R(h->c2r, (cufftComplex*)h->spec, h->real));
    k_pg_log<<<grid_of(frames * fr), 256, 0, st>>>(h->real, out, frames * fr);
    MM_LAUNCHED();
    return MM_OK;
}

void destroy(mm_pgn* h) {
    if (h->r2c) cufftDestroy(h->r2c);
    if (h->c2r) cufftDestroy(h->c2r);
    void* bufs[] = {h->H, h->spec, h->twx, h->twy, h->real};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete h;
}

int upload(void** dst, const void* src, size_t bytes, const char* what, size_t* ws) {
    MM_TRY(dev_alloc(dst, bytes, what));
    *ws += bytes;
    if (cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
        mm::set_error("mm_pgn_create: %s upload failed", what);
        return MM_ECUDA;
    }
    return MM_OK;
}

}  // namespace

extern "C" int mm_pgn_create(int n, int nz, int ntheta, const float* filt_host, mm_pgn** out) {
    MM_REQUIRE(out != nullptr, "mm_pgn_create: out is NULL");
    *out = nullptr;
    MM_REQUIRE(n >= 2 && n <= 65536 && nz >= 2 && nz <= 65536, "mm_pgn_create: n=%d, nz=%d out of range", n, nz);
    MM_REQUIRE(ntheta >= 1 && filt_host != nullptr, "mm_pgn_create: need ntheta >= 1 and the filter table");
    MM_CUDA(mmfft::init_constants());
    mm_pgn* h = new mm_pgn();
    h->n = n;
    h->nz = nz;
    h->ntheta = ntheta;
    h->nh = n / 2 + 1;
    // native line lengths: powers of two up to 4096, 3 * 2^k in [96, 3072]
    auto line_ok = [](int L) { return mm_is_pow2(L) ? L <= 4096 : (stockham::length_ok(L) && L >= 96 && L <= 3072); };
    h->native = line_ok(n) && line_ok(nz);
    auto fail = [&](int rc) {
        destroy(h);
        return rc;
    };
    int rc;
    if ((rc = upload((void**)&h->H, filt_host, (size_t)nz * h->nh * sizeof(float), "filter table", &h->ws_bytes)))
        return fail(rc);
    if ((rc = dev_alloc((void**)&h->spec, (size_t)ntheta * nz * h->nh * sizeof(float2), "Paganin spectra")))
        return fail(rc);
    h->ws_bytes += (size_t)ntheta * nz * h->nh * sizeof(float2);
    if (h->native) {
        std::vector<float2> tx(4 * (size_t)n, make_float2(0.f, 0.f)), ty(4 * (size_t)nz, make_float2(0.f, 0.f));
        stockham::host_twiddles(n, false, tx.data());
        stockham::host_twiddles(n, true, tx.data() + 2 * (size_t)n);
        stockham::host_twiddles(nz, false, ty.data());
        stockham::host_twiddles(nz, true, ty.data() + 2 * (size_t)nz);
        if ((rc = upload((void**)&h->twx, tx.data(), tx.size() * sizeof(float2), "x twiddles", &h->ws_bytes)) ||
            (rc = upload((void**)&h->twy, ty.data(), ty.size() * sizeof(float2), "y twiddles", &h->ws_bytes)))
            return fail(rc);
    } else {
        if ((rc = dev_alloc((void**)&h->real, (size_t)ntheta * nz * n * sizeof(float), "Paganin frames")))
            return fail(rc);
        h->ws_bytes += (size_t)ntheta * nz * n * sizeof(float);
        int dims[2] = {nz, n};
        if (cufftPlanMany(&h->r2c, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, ntheta) != CUFFT_SUCCESS ||
            cufftPlanMany(&h->c2r, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, ntheta) != CUFFT_SUCCESS) {
            mm::set_error("mm_pgn_create: cuFFT plan creation failed");
            return fail(MM_ECUFFT);
        }
    }
    *out = h;
    return MM_OK;
}

extern "C" int mm_pgn_destroy(mm_pgn* h) {
    if (!h) return MM_OK;
    cudaDeviceSynchronize();
    destroy(h);
    return MM_OK;
}

extern "C" int mm_pgn_retrieve(mm_pgn* h, const float* intensity, float* phase, int frames, void* stream) {
    MM_REQUIRE(h != nullptr, "mm_pgn_retrieve: NULL handle");
    MM_REQUIRE(intensity != nullptr && phase != nullptr, "mm_pgn_retrieve: NULL array");
    MM_REQUIRE(frames >= 1 && frames <= h->ntheta, "mm_pgn_retrieve: batch %d > cached ntheta %d", frames,
               h->ntheta);
    MM_RANGE(intensity, (size_t)frames * h->nz * h->n * 4, "mm_pgn_retrieve", "intensity");
    MM_RANGE(phase, (size_t)frames * h->nz * h->n * 4, "mm_pgn_retrieve", "phase");
    cudaStream_t st = (cudaStream_t)stream;
    if (!h->native) return run_general(h, intensity, phase, frames, st);
    const long rows = (long)frames * h->nz;
    MM_TRY(rows_pass(h, false, intensity, nullptr, rows, st));
    MM_TRY(cols_pass(h, frames, st));
    return rows_pass(h, true, nullptr, phase, rows, st);
}

extern "C" size_t mm_pgn_workspace_bytes(const mm_pgn* h) { return h ? h->ws_bytes : 0; }
