// Fresnel propagator D and its adjoint DT for sm_100a.
//
// Reference (processing/propagation.py:18-64, processing/kernels.py:530-550):
//   D(psi) = crop( IFFT2_unnorm( fker_j * FFT2( mirrorpad(psi) ) ) ),
//   fker_j = exp(-i pi lambda z_j (fx^2 + fy^2)) / (4 n nz).
// The chirp separates, K = Kx(fx) Ky(fy) (processing/propagation_large.py:7-13),
// and the y and x halves commute, so D runs as two passes over HBM:
//   y-pass  per column: mirror-pad to 2nz, FFT, *Ky/(2nz), IFFT, crop  -> mid
//   x-pass  per row:    mirror-pad to 2n,  FFT, *Kx/(2n),  IFFT, crop  -> out
// Each pass keeps its column/row in registers and shared memory
// (fft_smem.cuh): 24 bytes of HBM traffic per pixel for f32 in, c64 mid,
// f32 out.  psi = exp(-p s/beta_r) (cos p s, sin p s) (step3_propagation.py:
// 94-103) is built in the y-pass load and |u|^2 (:105-110) in the x-pass
// store.  The chirp phase is evaluated in FP64 and reduced mod 2 pi.
// DT is the exact adjoint: zero-embed, FFT, *conj(K), IFFT, fold the mirrored
// borders back onto their source pixels.
#include "mm_common.cuh"
#include "fft_smem.cuh"

#include <math.h>

#include <mutex>
#include <vector>

using mm::dev_alloc;
using mmfft::cmul;
using mmfft::cmulc;
using mmfft::reg_fft;
using mmfft::Split;

struct mm_prop {
    int n = 0, nz = 0, ntheta = 0, ndist = 0;
    float2* Kx = nullptr;   // (ndist, 2n)
    float2* Ky = nullptr;   // (ndist, 2nz)
    // Stockham pass twiddles of the 2n- and 2nz-point lines (fft_smem.cuh),
    // each in a 3L-entry slot (forward schedule, then reversed at 3L/2)
    float2* twx = nullptr;  // (3 * 2n)
    float2* twy = nullptr;  // (3 * 2nz)
    float2* mid = nullptr;  // (ntheta, nz, n)
    size_t ws_bytes = 0;
    mm::StageTimer tm;
};

namespace {

// Source index of padded position t (processing/kernels.py:541-544).
__device__ __forceinline__ int mirror_src(int t, int len) {
    const int h = len / 2;
    return t < h ? h - t - 1 : (t >= len + h ? 2 * len - t + h - 1 : t - h);
}
// The second padded position that folds onto pixel r (the first is r + len/2).
__device__ __forceinline__ int mirror_partner(int r, int len) {
    const int h = len / 2;
    return r < h ? h - 1 - r : 2 * len + h - 1 - r;
}

// ---------------------------------------------------------------- y-pass
// IN: 0 complex psi, 1 real projection (psi built on load).  Block (CW, G):
// lanes run over CW adjacent columns, threadIdx.y over the G = 2nz/16
// threads of each column's Stockham transform (fft_smem.cuh).
template <int L, int CW, int IN, bool ADJ>
__global__ void __launch_bounds__(CW * stockham::Sched<L>::G, 1024 / (CW * stockham::Sched<L>::G)) k_ypass(const void* __restrict__ src,
                                                                       float2* __restrict__ dst,
                                                                       const float2* __restrict__ Ky,
                                                                       const float2* __restrict__ tw, int n, int nz,
                                                                       float s, float ib) {
    using S = stockham::Sched<L>;
    extern __shared__ float2 sm[];  // buf [L][CW], then staged rows [nz][CW]
    float2* buf = sm;
    float2* stg = sm + L * CW;
    const int c = threadIdx.x, g = threadIdx.y;
    const int x = blockIdx.x * CW + c;
    const bool live = x < n;
    const long plane = (long)blockIdx.y * nz * n;
    // stage the nz source rows of this column block once (psi built here);
    // the mirror padding then reads each of them twice from shared memory
    for (int r = g; r < nz; r += S::G) {
        float2 a = make_float2(0.f, 0.f);
        if (live) {
            const long off = plane + (long)r * n + x;
            if (IN == 0) {
                a = __ldg(static_cast<const float2*>(src) + off);
            } else {
                const float ph = __ldg(static_cast<const float*>(src) + off) * s;
                const float at = expf(-ph * ib);
                float sn, cs;
                sincosf(ph, &sn, &cs);
                a = make_float2(at * cs, at * sn);
            }
        }
        stg[r * CW + c] = a;
    }
    __syncthreads();
    const stockham::ColAddr<CW> ad{c};
    auto ld_in = [&](int pos) -> float2 {
        if (!ADJ) return stg[mirror_src(pos, nz) * CW + c];
        const int r = pos - nz / 2;
        return (r >= 0 && r < nz) ? stg[r * CW + c] : make_float2(0.f, 0.f);
    };
    auto mul = [&](int pos, float2 v) -> float2 {
        const float2 K = __ldg(Ky + pos);
        return ADJ ? cmulc(v, K) : cmul(v, K);
    };
    const float2* twf = tw;
    const float2* twi = tw + 3 * L / 2;
    if (!ADJ) {
        auto st_out = [&](int pos, float2 v) {
            const int r = pos - nz / 2;
            if (live && r >= 0 && r < nz) dst[plane + (long)r * n + x] = v;
        };
        stockham::conv<L>(buf, ad, ld_in, mul, st_out, g, twf, twi);
    } else {
        auto st_b = [&](int pos, float2 v) { buf[pos * CW + c] = v; };
        stockham::conv<L>(buf, ad, ld_in, mul, st_b, g, twf, twi);
        __syncthreads();
        for (int r = g; r < nz; r += S::G) {
            const float2 a = buf[(r + nz / 2) * CW + c], b = buf[mirror_partner(r, nz) * CW + c];
            if (live) dst[plane + (long)r * n + x] = make_float2(a.x + b.x, a.y + b.y);
        }
    }
}

// ---------------------------------------------------------------- x-pass
// OUT: 0 complex, 1 |.|^2 float, 2 (forward, gradient of the L2 loss):
// g = 4 (|u|^2 - d) u with d = aux, plus per-block sums of (|u|^2 - d)^2
// in partials[blockIdx.x]; 3 (adjoint, chain through psi): dL/dp =
// s Re(conj(g) (i - ib) psi(p)) with p = aux, psi(p) = exp(-p s ib)(cos p s,
// sin p s), written as float.  Block (G, RPB): G = 2n/16 threads per row.
template <int L, int RPB, int OUT, bool ADJ>
__global__ void __launch_bounds__(RPB * stockham::Sched<L>::G, 512 / (RPB * stockham::Sched<L>::G)) k_xpass(const float2* __restrict__ src,
                                                                        void* __restrict__ dst,
                                                                        const float2* __restrict__ Kx,
                                                                        const float2* __restrict__ tw, int n,
                                                                        long rows, const float* __restrict__ aux,
                                                                        float* __restrict__ partials, float s,
                                                                        float ib) {
    extern __shared__ float2 sm[];  // [RPB][L + L/16]
    constexpr int LP = L + L / 16;
    const int g = threadIdx.x, rr = threadIdx.y;
    const long row = (long)blockIdx.x * RPB + rr;
    const bool live = row < rows;
    const stockham::RowAddr ad{rr * LP};
    float2* buf = sm;
    const float2* in = src + row * n;
    auto ld_in = [&](int pos) -> float2 {
        int col = ADJ ? pos - n / 2 : mirror_src(pos, n);
        if (ADJ && (col < 0 || col >= n)) return make_float2(0.f, 0.f);
        return live ? __ldg(in + col) : make_float2(0.f, 0.f);
    };
    auto mul = [&](int pos, float2 v) -> float2 {
        const float2 K = __ldg(Kx + pos);
        return ADJ ? cmulc(v, K) : cmul(v, K);
    };
    const float2* twf = tw;
    const float2* twi = tw + 3 * L / 2;
    if (!ADJ) {
        float lsum = 0.f;
        auto st_out = [&](int pos, float2 v) {
            const int c = pos - n / 2;
            if (live && c >= 0 && c < n) {
                if (OUT == 0) {
                    static_cast<float2*>(dst)[row * n + c] = v;
                } else if (OUT == 1) {
                    static_cast<float*>(dst)[row * n + c] = v.x * v.x + v.y * v.y;
                } else {
                    const float r = v.x * v.x + v.y * v.y - __ldg(aux + row * n + c);
                    lsum = fmaf(r, r, lsum);
                    static_cast<float2*>(dst)[row * n + c] = make_float2(4.f * r * v.x, 4.f * r * v.y);
                }
            }
        };
        stockham::conv<L>(buf, ad, ld_in, mul, st_out, g, twf, twi);
        if (OUT == 2) {  // deterministic block sum of the squared residuals
            __syncthreads();
            float* red = reinterpret_cast<float*>(sm);
            for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
            const int tid = rr * blockDim.x + g, nw = (blockDim.x * blockDim.y + 31) / 32;
            if ((tid & 31) == 0) red[tid >> 5] = lsum;
            __syncthreads();
            if (tid == 0) {
                float t = 0.f;
                for (int w = 0; w < nw; ++w) t += red[w];
                partials[blockIdx.x] = t;
            }
        }
    } else {
        auto st_b = [&](int pos, float2 v) { buf[ad(pos)] = v; };
        stockham::conv<L>(buf, ad, ld_in, mul, st_b, g, twf, twi);
        __syncthreads();
        for (int c = g; c < n; c += stockham::Sched<L>::G) {
            const float2 a = buf[ad(c + n / 2)], b = buf[ad(mirror_partner(c, n))];
            if (!live) continue;
            const float2 gv = make_float2(a.x + b.x, a.y + b.y);
            if (OUT == 3) {
                const float ph = __ldg(aux + row * n + c) * s;
                const float at = expf(-ph * ib);
                float sn, cs;
                sincosf(ph, &sn, &cs);
                const float px = at * cs, py = at * sn;              // psi
                const float wx = -ib * px - py, wy = px - ib * py;   // (i - ib) psi
                static_cast<float*>(dst)[row * n + c] = s * (gv.x * wx + gv.y * wy);
            } else {
                static_cast<float2*>(dst)[row * n + c] = gv;
            }
        }
    }
}

// ---------------------------------------------------------------- launch
template <int L, int IN, bool ADJ>
int launch_y(mm_prop* h, const void* src, int ntheta, int j, float s, float ib, cudaStream_t st) {
    constexpr int G = stockham::Sched<L>::G;
    constexpr int CW0 = 256 / G;
    constexpr int CW = CW0 < 4 ? 4 : (CW0 > 32 ? 32 : CW0);
    const size_t smem = (size_t)(L * CW + (L / 2) * CW) * sizeof(float2);
    auto kern = k_ypass<L, CW, IN, ADJ>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 block(CW, G), grid((h->n + CW - 1) / CW, ntheta);
    h->tm.begin(0, st);
    kern<<<grid, block, smem, st>>>(src, h->mid, h->Ky + (size_t)j * 2 * h->nz, h->twy, h->n, h->nz, s, ib);
    MM_LAUNCHED();
    h->tm.end(st, 1);
    return MM_OK;
}

template <int L, int OUT, bool ADJ>
int launch_x(mm_prop* h, void* dst, int ntheta, int j, cudaStream_t st, const float* aux = nullptr,
             float* partials = nullptr, float s = 0.f, float ib = 0.f) {
    constexpr int G = stockham::Sched<L>::G;
    constexpr int RPB = G >= 256 ? 1 : 256 / G;
    const size_t smem = (size_t)RPB * (L + L / 16) * sizeof(float2);
    auto kern = k_xpass<L, RPB, OUT, ADJ>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long rows = (long)ntheta * h->nz;
    dim3 block(G, RPB), grid((unsigned)((rows + RPB - 1) / RPB));
    h->tm.begin(1, st);
    kern<<<grid, block, smem, st>>>(h->mid, dst, h->Kx + (size_t)j * 2 * h->n, h->twx, h->n, rows, aux, partials,
                                    s, ib);
    MM_LAUNCHED();
    h->tm.end(st, 1);
    return MM_OK;
}

template <int IN, bool ADJ>
int dispatch_y(mm_prop* h, const void* src, int ntheta, int j, float s, float ib, cudaStream_t st) {
    switch (2 * h->nz) {
        case 4: return launch_y<4, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 8: return launch_y<8, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 16: return launch_y<16, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 32: return launch_y<32, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 64: return launch_y<64, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 128: return launch_y<128, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 256: return launch_y<256, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 512: return launch_y<512, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 1024: return launch_y<1024, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 2048: return launch_y<2048, IN, ADJ>(h, src, ntheta, j, s, ib, st);
        case 4096: return launch_y<4096, IN, ADJ>(h, src, ntheta, j, s, ib, st);
    }
    MM_REQUIRE(false, "unsupported 2*nz=%d", 2 * h->nz);
}

template <int OUT, bool ADJ>
int dispatch_x(mm_prop* h, void* dst, int ntheta, int j, cudaStream_t st, const float* aux = nullptr,
               float* partials = nullptr, float s = 0.f, float ib = 0.f) {
    switch (2 * h->n) {
        case 4: return launch_x<4, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 8: return launch_x<8, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 16: return launch_x<16, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 32: return launch_x<32, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 64: return launch_x<64, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 128: return launch_x<128, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 256: return launch_x<256, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 512: return launch_x<512, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 1024: return launch_x<1024, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 2048: return launch_x<2048, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
        case 4096: return launch_x<4096, OUT, ADJ>(h, dst, ntheta, j, st, aux, partials, s, ib);
    }
    MM_REQUIRE(false, "unsupported 2*n=%d", 2 * h->n);
}

int check_call(const mm_prop* h, const void* a, const void* b, int ntheta, int j, const char* who) {
    MM_REQUIRE(h != nullptr, "%s: NULL handle", who);
    MM_REQUIRE(a != nullptr && b != nullptr, "%s: NULL array", who);
    MM_REQUIRE(ntheta >= 1 && ntheta <= h->ntheta, "%s: ntheta=%d outside [1, %d]", who, ntheta, h->ntheta);
    MM_REQUIRE(j >= 0 && j < h->ndist, "%s: distance index %d outside [0, %d)", who, j, h->ndist);
    return MM_OK;
}

void destroy(mm_prop* h) {
    h->tm.release();
    void* bufs[] = {h->Kx, h->Ky, h->twx, h->twy, h->mid};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete h;
}

// exp(-i pi lambda z f^2) / len for the float32 fftfreq grid of `len` points
// (processing/propagation.py:23-31), phase in FP64 reduced mod 2 pi.
void chirp(std::vector<float2>& out, int len, double voxelsize, double wavelength, double z) {
    const double val = 1.0 / (len * voxelsize);
    for (int k = 0; k < len; ++k) {
        const int kk = k < (len + 1) / 2 ? k : k - len;
        const double f = (double)(float)(kk * val);
        double ph = fmod(M_PI * wavelength * z * f * f, 2.0 * M_PI);
        out[k] = make_float2((float)(cos(-ph) / len), (float)(sin(-ph) / len));
    }
}

// Stockham twiddle tables of a length-len line (fft_smem.cuh) in a 3*len
// slot: the forward schedule's at 0, the reversed schedule's at 3*len/2.
void twiddles(std::vector<float2>& out, int len) {
    out.assign(3 * (size_t)len, make_float2(0.f, 0.f));
    stockham::host_twiddles(len, false, out.data());
    stockham::host_twiddles(len, true, out.data() + 3 * len / 2);
}

}  // namespace

extern "C" int mm_prop_create(int n, int nz, int ntheta, int ndist, double wavelength, double voxelsize,
                              const double* distance_host, mm_prop** out) {
    MM_REQUIRE(out != nullptr, "mm_prop_create: out is NULL");
    *out = nullptr;
    MM_REQUIRE(mm_is_pow2(2L * n) && 2 * n >= 4 && 2 * n <= 4096,
               "mm_prop_create: 2n=%d must be a power of two in [4, 4096]", 2 * n);
    MM_REQUIRE(mm_is_pow2(2L * nz) && 2 * nz >= 4 && 2 * nz <= 4096,
               "mm_prop_create: 2nz=%d must be a power of two in [4, 4096]", 2 * nz);
    MM_REQUIRE(ntheta >= 1 && ndist >= 1 && distance_host != nullptr, "mm_prop_create: bad ntheta/ndist");
    MM_REQUIRE(voxelsize > 0, "mm_prop_create: voxelsize must be positive");
    MM_CUDA(mmfft::init_constants());
    mm_prop* h = new mm_prop();
    h->n = n;
    h->nz = nz;
    h->ntheta = ntheta;
    h->ndist = ndist;
    std::vector<float2> kx((size_t)ndist * 2 * n), ky((size_t)ndist * 2 * nz), tx, ty, tmp;
    for (int j = 0; j < ndist; ++j) {
        tmp.assign(2 * n, make_float2(0, 0));
        chirp(tmp, 2 * n, voxelsize, wavelength, distance_host[j]);
        std::copy(tmp.begin(), tmp.end(), kx.begin() + (size_t)j * 2 * n);
        tmp.assign(2 * nz, make_float2(0, 0));
        chirp(tmp, 2 * nz, voxelsize, wavelength, distance_host[j]);
        std::copy(tmp.begin(), tmp.end(), ky.begin() + (size_t)j * 2 * nz);
    }
    twiddles(tx, 2 * n);
    twiddles(ty, 2 * nz);
    struct B { float2** p; const std::vector<float2>* v; const char* what; } bs[] = {
        {&h->Kx, &kx, "x chirp"}, {&h->Ky, &ky, "y chirp"}, {&h->twx, &tx, "x twiddles"}, {&h->twy, &ty, "y twiddles"}};
    for (auto& b : bs) {
        int rc = dev_alloc((void**)b.p, b.v->size() * sizeof(float2), b.what);
        if (rc != MM_OK) {
            destroy(h);
            return rc;
        }
        h->ws_bytes += b.v->size() * sizeof(float2);
        if (cudaMemcpy(*b.p, b.v->data(), b.v->size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
            mm::set_error("mm_prop_create: table upload failed");
            destroy(h);
            return MM_ECUDA;
        }
    }
    const size_t mid = (size_t)ntheta * nz * n;
    int rc = dev_alloc((void**)&h->mid, mid * sizeof(float2), "propagator intermediate");
    if (rc != MM_OK) {
        destroy(h);
        return rc;
    }
    h->ws_bytes += mid * sizeof(float2);
    *out = h;
    return MM_OK;
}

extern "C" int mm_prop_destroy(mm_prop* h) {
    if (!h) return MM_OK;
    cudaDeviceSynchronize();
    destroy(h);
    return MM_OK;
}

extern "C" int mm_prop_D(mm_prop* h, const void* psi, void* out, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, psi, out, ntheta, j, "mm_prop_D"));
    cudaStream_t st = (cudaStream_t)stream;
    MM_TRY((dispatch_y<0, false>(h, psi, ntheta, j, 0.f, 0.f, st)));
    return dispatch_x<0, false>(h, out, ntheta, j, st);
}

extern "C" int mm_prop_DT(mm_prop* h, const void* g, void* out, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, g, out, ntheta, j, "mm_prop_DT"));
    cudaStream_t st = (cudaStream_t)stream;
    MM_TRY((dispatch_y<0, true>(h, g, ntheta, j, 0.f, 0.f, st)));
    return dispatch_x<0, true>(h, out, ntheta, j, st);
}

extern "C" int mm_prop_intensity(mm_prop* h, const float* proj, float inv_norm, float inv_beta_ratio,
                                 float* intensity, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, proj, intensity, ntheta, j, "mm_prop_intensity"));
    cudaStream_t st = (cudaStream_t)stream;
    MM_TRY((dispatch_y<1, false>(h, proj, ntheta, j, inv_norm, inv_beta_ratio, st)));
    return dispatch_x<1, false>(h, intensity, ntheta, j, st);
}

extern "C" int mm_prop_set_timing(mm_prop* h, int on) {
    MM_REQUIRE(h != nullptr, "mm_prop_set_timing: NULL handle");
    h->tm.reset();
    h->tm.on = on != 0;
    return MM_OK;
}

extern "C" int mm_prop_get_timing(mm_prop* h, double* ms, long long* calls, int nstages, long long* kernels) {
    MM_REQUIRE(h != nullptr, "mm_prop_get_timing: NULL handle");
    h->tm.read();
    for (int i = 0; i < nstages && i < mm::StageTimer::kMax; ++i) {
        if (ms) ms[i] = h->tm.ms[i];
        if (calls) calls[i] = h->tm.calls[i];
    }
    if (kernels) *kernels = h->tm.kernels;
    return MM_OK;
}

// ==========================================================================
// Allocation-free Fresnel D.
//
// Some callers cannot allocate device memory at call time: a host program
// whose GPU memory is entirely reserved up front by its own pool allocator
// (an acquisition or streaming-reconstruction service, or a process where
// another framework's caching allocator owns the device) sees cudaMalloc fail
// or stall other work once it is running.  mm_prop_D_noalloc serves them: it
// takes no handle and calls no cudaMalloc/cudaFree or allocating library
// routine.  Its working memory -- the chirp and twiddle tables and the
// column-pass intermediate -- lives in the file-scope array below, which
// every GPU that loads this library holds (kNoAllocBytes) until the process
// exits.  All calls share that one array and it keeps the last call's
// contents, so calls that overlap on the GPU (two streams, two host threads)
// race; callers must order them.  Nothing in it needs to start at zero: every
// call rewrites the tables and the intermediate before reading them.
static constexpr size_t kNoAllocBytes = 64ull << 20;  // 64 MiB per device
static __device__ __align__(256) float2 g_noalloc_scratch[kNoAllocBytes / sizeof(float2)];

namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};

// Per-device set-up, done by the first call on each device (with that device
// current): resolve the array's device address and upload the FFT constants.
int noalloc_setup(float2** out) {
    int dev = 0;
    MM_CUDA(cudaGetDevice(&dev));
    MM_REQUIRE(dev >= 0 && dev < 64, "mm_prop_D_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            mm::set_error("mm_prop_D_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return MM_ECUDA;
        }
        MM_CUDA(mmfft::init_constants());
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<float2*>(g_noalloc_ptr[dev]);
    return MM_OK;
}

// Chirp and twiddle tables of one distance, computed on the device in FP64
// exactly as chirp() / twiddles() do on the host for mm_prop_create.
__global__ void k_noalloc_tables(float2* __restrict__ Kx, float2* __restrict__ Ky, float2* __restrict__ twx,
                                 float2* __restrict__ twy, int n, int nz, double wavelength, double voxelsize,
                                 double z) {
    const int total = 2 * n + 2 * nz + 6 * n + 6 * nz;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int i = t;
        if (i < 2 * n + 2 * nz) {  // chirp along x then y
            const bool along_x = i < 2 * n;
            const int len = along_x ? 2 * n : 2 * nz;
            const int k = along_x ? i : i - 2 * n;
            const double val = 1.0 / (len * voxelsize);
            const int kk = k < (len + 1) / 2 ? k : k - len;
            const double f = (double)(float)(kk * val);
            const double ph = fmod(M_PI * wavelength * z * f * f, 2.0 * M_PI);
            const float2 w = make_float2((float)(cos(-ph) / len), (float)(sin(-ph) / len));
            if (along_x) Kx[k] = w; else Ky[k] = w;
            continue;
        }
        i -= 2 * n + 2 * nz;  // twiddles: x slot (3 * 2n) then y slot (3 * 2nz)
        const bool along_x = i < 6 * n;
        const int len = along_x ? 2 * n : 2 * nz;
        int q = along_x ? i : i - 6 * n;
        float2* tab = along_x ? twx : twy;
        const int slot_q = q;
        const bool rev = q >= 3 * len / 2;
        if (rev) q -= 3 * len / 2;
        // entry q of stockham::host_twiddles(len, rev, .)
        int P = 1;
        if (len > 16) {
            int lg = 0;
            while ((1 << lg) < len) ++lg;
            P = (lg + 3) / 4;
        }
        const int small = len >> (4 * (P - 1));
        int o = 0, ns = rev ? small : (P > 1 ? 16 : small);
        float2 w = make_float2(0.f, 0.f);
        for (int p = 1; p < P; ++p) {
            const int rp = rev ? 16 : (p < P - 1 ? 16 : small);
            if (q >= o && q < o + ns * rp) {
                const int ii = (q - o) / ns, k = (q - o) % ns;
                double sv, cv;
                sincospi(-2.0 * (double)(((long)ii * k) % (ns * rp)) / (ns * rp), &sv, &cv);
                w = make_float2((float)cv, (float)sv);
            }
            o += ns * rp;
            ns *= rp;
        }
        tab[slot_q] = w;
    }
}

}  // namespace

extern "C" int mm_prop_D_noalloc(int n, int nz, int ntheta, double wavelength, double voxelsize, double distance,
                                 const void* psi, void* out, void* stream) {
    MM_REQUIRE(psi != nullptr && out != nullptr, "mm_prop_D_noalloc: NULL array");
    MM_REQUIRE(mm_is_pow2(2L * n) && 2 * n >= 4 && 2 * n <= 4096,
               "mm_prop_D_noalloc: 2n=%d must be a power of two in [4, 4096]", 2 * n);
    MM_REQUIRE(mm_is_pow2(2L * nz) && 2 * nz >= 4 && 2 * nz <= 4096,
               "mm_prop_D_noalloc: 2nz=%d must be a power of two in [4, 4096]", 2 * nz);
    MM_REQUIRE(ntheta >= 1 && voxelsize > 0, "mm_prop_D_noalloc: bad ntheta/voxelsize");
    const size_t tables = (size_t)8 * n + 8 * nz;
    const size_t need = (tables + (size_t)ntheta * nz * n) * sizeof(float2);
    MM_REQUIRE(need <= kNoAllocBytes,
               "mm_prop_D_noalloc: ntheta*nz*n=%zu needs %zu bytes of scratch, more than the %zu-byte "
               "static buffer (use mm_prop_D, or fewer angles per call)",
               (size_t)ntheta * nz * n, need, kNoAllocBytes);
    float2* base = nullptr;
    MM_TRY(noalloc_setup(&base));
    cudaStream_t st = (cudaStream_t)stream;
    mm_prop h;  // view onto the static scratch; owns nothing
    h.n = n;
    h.nz = nz;
    h.ntheta = ntheta;
    h.ndist = 1;
    h.Kx = base;
    h.Ky = h.Kx + 2 * n;
    h.twx = h.Ky + 2 * nz;
    h.twy = h.twx + 6 * n;
    h.mid = h.twy + 6 * nz;
    k_noalloc_tables<<<(unsigned)((tables + 255) / 256), 256, 0, st>>>(h.Kx, h.Ky, h.twx, h.twy, n, nz, wavelength,
                                                                      voxelsize, distance);
    MM_LAUNCHED();
    MM_TRY((dispatch_y<0, false>(&h, psi, ntheta, 0, 0.f, 0.f, st)));
    return dispatch_x<0, false>(&h, out, ntheta, 0, st);
}

extern "C" long mm_prop_grad_partials(mm_prop* h, int ntheta) {
    if (!h || ntheta < 1) return 0;
    const int G = (2 * h->n) >= 16 ? (2 * h->n) / 16 : 1;
    const int rpb = G >= 256 ? 1 : 256 / G;
    return ((long)ntheta * h->nz + rpb - 1) / rpb;
}

extern "C" int mm_prop_grad_forward(mm_prop* h, const float* proj, const float* data, float inv_norm,
                                    float inv_beta_ratio, void* gu, float* partials, int ntheta, int j,
                                    void* stream) {
    MM_TRY(check_call(h, proj, gu, ntheta, j, "mm_prop_grad_forward"));
    MM_REQUIRE(data != nullptr && partials != nullptr, "mm_prop_grad_forward: NULL data/partials");
    cudaStream_t st = (cudaStream_t)stream;
    MM_TRY((dispatch_y<1, false>(h, proj, ntheta, j, inv_norm, inv_beta_ratio, st)));
    return dispatch_x<2, false>(h, gu, ntheta, j, st, data, partials, inv_norm, inv_beta_ratio);
}

extern "C" int mm_prop_grad_backward(mm_prop* h, const void* gu, const float* proj, float inv_norm,
                                     float inv_beta_ratio, float* gp, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, gu, gp, ntheta, j, "mm_prop_grad_backward"));
    MM_REQUIRE(proj != nullptr, "mm_prop_grad_backward: NULL proj");
    cudaStream_t st = (cudaStream_t)stream;
    MM_TRY((dispatch_y<0, true>(h, gu, ntheta, j, 0.f, 0.f, st)));
    return dispatch_x<3, true>(h, gp, ntheta, j, st, proj, nullptr, inv_norm, inv_beta_ratio);
}
