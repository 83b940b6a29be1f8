// Fresnel propagator D and its adjoint DT for sm_100a.
//
// Reference (processing/propagation.py:18-64, processing/kernels.py:530-550):
//   D(psi) = crop( IFFT2_unnorm( fker_j * FFT2( mirrorpad(psi) ) ) ),
//   fker_j = exp(-i pi lambda z_j (fx^2 + fy^2)) / (4 n nz).
// The chirp separates, K = Kx(fx) Ky(fy) (processing/propagation_large.py:7-13),
// and the y and x halves commute, so D runs as two passes over HBM: a column
// pass along y (length nz) and a row pass along x (length n).
//
// Half-length lines.  The padding repeats the edge sample (kernels.py:541-544),
// so the 2N-point padded line is the even, half-sample-symmetric extension of
// the N input samples, and the chirp is even in frequency (K[k] = K[2N-k]).
// Pad -> FFT_2N -> *K -> IFFT_2N -> crop is then exactly
// DCT-III . diag(K[0..N)) . DCT-II on the N samples, and both DCTs run on
// N-point complex FFTs (Makhoul's reordering, IEEE TASSP 28(1), 1980):
//   v[p] = a[sig(p)],  sig(p) = 2p (p < N/2), 2N-1-2p (p >= N/2)
//   V = FFT_N(v)
//   W[k] = P[k] V[k] + Q[k] V[(N-k) mod N]
//   out[sig(p)] = IFFT_N,unnorm(W)[p]
// with, for the chirp Kh = K/(2N) of the 2N grid and Kh' = Kh[N-k] (Kh[0]
// at k = 0):  P[k] = Kh[k] + Kh',  Q[k] = e^{i pi k/N} (Kh[k] - Kh')
// (Q[0] = 0).  The operator is complex symmetric, so the adjoint DT is the
// same line transform with conj(K): no zero embedding and no border fold.
// Per pixel: f32 in, c64 intermediate, f32 out (24 bytes of HBM traffic);
// psi = exp(-p s/beta_r)(cos p s, sin p s) (step3_propagation.py:94-103) is
// built in the column-pass load and |u|^2 (:105-110) in the row-pass store.
// Chirp phases and the P/Q tables are evaluated in FP64 (phase mod 2 pi).
//
// General sizes.  The identity holds for every N (with the split point of
// sig at ceil(N/2)), so sizes outside the fused kernels' range (n or nz not a
// power of two in [2, 2048]) run the same algebra in 2-D: a reordering load
// (psi on load), one cuFFT 2-D transform per frame, the tensor-product pair
// step W = (Py + Qy Ry)(Px + Qx Rx) V with R the reflection k -> N-k, the
// inverse transform and a reordering store (|.|^2 or the loss terms).
#include "mm_common.cuh"
#include "fft_smem.cuh"

#include <math.h>

#include <algorithm>
#include <mutex>
#include <vector>

using mm::dev_alloc;
using mmfft::cmul;
using mmfft::cmulc;

struct mm_prop {
    int n = 0, nz = 0, ntheta = 0, ndist = 0;
    // per distance, P/Q line tables as float4 (P.re, P.im, Q.re, Q.im):
    // [dist][0][k] for D, [dist][1][k] for DT
    float4* Sx = nullptr;   // (ndist, 2, n)
    float4* Sy = nullptr;   // (ndist, 2, nz)
    // Stockham pass twiddles of the n- and nz-point lines (fft_smem.cuh),
    // each in a 3N-entry slot (forward schedule, then reversed at 3N/2)
    float2* twx = nullptr;  // (3 * n)
    float2* twy = nullptr;  // (3 * nz)
    float2* mid = nullptr;  // (ntheta, nz, n)
    // general sizes: second frame buffer and cuFFT 2-D plans (ntheta frames,
    // and the last smaller batch used)
    bool general = false;
    float2* mid2 = nullptr;
    cufftHandle plan_full = 0, plan_part = 0;
    int part_batch = 0;
    size_t ws_bytes = 0;
    mm::StageTimer tm;
};

namespace {

// Makhoul order: line position p holds sample sig(p).
__device__ __forceinline__ int sig(int p, int N) { return p < (N + 1) / 2 ? 2 * p : 2 * N - 1 - 2 * p; }

__device__ __forceinline__ float2 pair_mix(const float4* __restrict__ S, int k, float2 a, float2 b) {
    const float4 pq = __ldg(S + k);
    const float2 pa = cmul(a, make_float2(pq.x, pq.y));
    const float2 qb = cmul(b, make_float2(pq.z, pq.w));
    return make_float2(pa.x + qb.x, pa.y + qb.y);
}

// ---------------------------------------------------------------- y-pass
// IN: 0 complex input, 1 real projection (psi built on load).  Block
// (CW, G): lanes run over CW adjacent columns, threadIdx.y over the
// G = nz/16 threads of each column's Stockham transform (fft_smem.cuh).
// NXC: the row length n fixed at compile time (row offsets become immediates), 0 for runtime.
template <int N, int CW, int IN, int NXC>
__global__ void __launch_bounds__(CW * stockham::Sched<N>::G,
                                  (stockham::Sched<N>::P2 ? 1024 : 512) / (CW * stockham::Sched<N>::G))
    k_ypass(const void* __restrict__ src, float2* __restrict__ dst, const float4* __restrict__ Sy,
            const float2* __restrict__ tw, int n_rt, float s, float ib) {
    const int n = NXC > 0 ? NXC : n_rt;
    extern __shared__ float2 sm[];  // [rows(N)][CW]
    const int c = threadIdx.x, g = threadIdx.y;
    const int x = blockIdx.x * CW + c;
    const bool live = x < n;
    const long plane = (long)blockIdx.y * N * n;
    const stockham::ColAddr<CW> ad{c};
    auto ld = [&](int pos) -> float2 {
        if (!live) return make_float2(0.f, 0.f);
        const long off = plane + (long)sig(pos, N) * n + x;
        if (IN == 0) return __ldg(static_cast<const float2*>(src) + off);
        const float ph = __ldg(static_cast<const float*>(src) + off) * s;
        const float at = expf(-ph * ib);
        float sn, cs;
        sincosf(ph, &sn, &cs);
        return make_float2(at * cs, at * sn);
    };
    auto pair = [&](int k, float2 a, float2 b) { return pair_mix(Sy, k, a, b); };
    auto st = [&](int pos, float2 v) {
        if (live) dst[plane + (long)sig(pos, N) * n + x] = v;
    };
    stockham::pairconv<N>(sm, ad, ld, pair, st, g, tw, tw + 3 * N / 2);
}

// The column pass for 64-row frames (IN 1: psi built on load from the
// projections; IN 0: complex input), persistent and software-pipelined: each
// block walks over (frame, 32-column group) items and loads the next item's
// 16 input values per thread before it transforms the current one, so the
// loads of one item overlap the FFT of the previous (the one-item-per-block
// form waits on its loads at the start of every item).
template <int IN>
struct ColIn;
template <>
struct ColIn<0> { using T = float2; };
template <>
struct ColIn<1> { using T = float; };

// Columns per block of the prefetching column pass (a block of CW x G
// threads, 128 or 256).
template <int N>
constexpr int pf_cols() {
    return stockham::Sched<N>::G >= 32 ? 256 / stockham::Sched<N>::G : 128 / stockham::Sched<N>::G;
}

template <int N, int IN, int NXC>
__global__ void __launch_bounds__(pf_cols<N>() * stockham::Sched<N>::G,
                                  (IN == 1 ? 896 : 640) / (pf_cols<N>() * stockham::Sched<N>::G))
    k_ypass_pf(const void* __restrict__ src_v, float2* __restrict__ dst, const float4* __restrict__ Sy,
               const float2* __restrict__ tw, long items, int n_rt, float s, float ib) {
    using T = typename ColIn<IN>::T;
    constexpr int CW = pf_cols<N>(), NG = stockham::PassShape<N, false, 0>::NG;
    static_assert(stockham::Sched<N>::V == 16 && stockham::PassShape<N, false, 0>::RP == 16 &&
                      stockham::PassShape<N, false, 0>::Q == 1,
                  "first pass: radix 16, one group per thread");
    const T* __restrict__ src = static_cast<const T*>(src_v);
    const int n = NXC > 0 ? NXC : n_rt;
    extern __shared__ float2 sm[];
    const int c = threadIdx.x, g = threadIdx.y;
    const int ngroups = n / CW;
    const stockham::ColAddr<CW> ad{c};
    T raw[16], nxt[16];
    auto fetch = [&](long it, T (&v)[16]) {
        const long frame = it / ngroups;
        const int x = (int)(it % ngroups) * CW + c;
        const T* base = src + frame * N * (long)n + x;
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = __ldg(base + (long)sig(g + NG * i, N) * n);
    };
    long it = blockIdx.x;
    if (it < items) fetch(it, raw);
    for (; it < items; it += gridDim.x) {
        const long next = it + gridDim.x;
        if (next < items) fetch(next, nxt);
        const long frame = it / ngroups;
        const int x = (int)(it % ngroups) * CW + c;
        const long plane = frame * N * (long)n;
        auto ld = [&](int pos) -> float2 {
            if constexpr (IN == 0) {
                return raw[(pos - g) / NG];
            } else {
                const float ph = raw[(pos - g) / NG] * s;
                const float at = expf(-ph * ib);
                float sn, cs;
                sincosf(ph, &sn, &cs);
                return make_float2(at * cs, at * sn);
            }
        };
        auto pair = [&](int k, float2 a, float2 b) { return pair_mix(Sy, k, a, b); };
        auto st = [&](int pos, float2 v) { dst[plane + (long)sig(pos, N) * n + x] = v; };
        stockham::pairconv<N>(sm, ad, ld, pair, st, g, tw, tw + 3 * N / 2);
        __syncthreads();  // the next item reuses sm
#pragma unroll
        for (int i = 0; i < 16; ++i) raw[i] = nxt[i];
    }
}

// ---------------------------------------------------------------- x-pass
// OUT: 0 complex, 1 |.|^2 float, 2 (forward, gradient of the L2 loss):
// g = 4 (|u|^2 - d) u with d = aux, plus per-block sums of (|u|^2 - d)^2
// in partials[blockIdx.x]; 3 (adjoint, chain through psi): dL/dp =
// s Re(conj(g) (i - ib) psi(p)) with p = aux, psi(p) = exp(-p s ib)(cos p s,
// sin p s), written as float.  Block (G, RPB): G = n/16 threads per row.
template <int N, int RPB, int OUT>
__global__ void __launch_bounds__(RPB * stockham::Sched<N>::G, 512 / (RPB * stockham::Sched<N>::G))
    k_xpass(const float2* __restrict__ src, void* __restrict__ dst, const float4* __restrict__ Sx,
            const float2* __restrict__ tw, long rows, const float* __restrict__ aux, float* __restrict__ partials,
            float s, float ib) {
    extern __shared__ float2 sm[];  // [RPB][N + N/16]
    constexpr int LP = N + N / 16;
    const int g = threadIdx.x, rr = threadIdx.y;
    const long row = (long)blockIdx.x * RPB + rr;
    const bool live = row < rows;
    const stockham::RowAddr ad{rr * LP};
    const float2* in = src + row * N;
    auto ld = [&](int pos) -> float2 { return live ? __ldg(in + sig(pos, N)) : make_float2(0.f, 0.f); };
    auto pair = [&](int k, float2 a, float2 b) { return pair_mix(Sx, k, a, b); };
    float lsum = 0.f;
    auto st = [&](int pos, float2 v) {
        if (!live) return;
        const long o = row * N + sig(pos, N);
        if (OUT == 0) {
            static_cast<float2*>(dst)[o] = v;
        } else if (OUT == 1) {
            static_cast<float*>(dst)[o] = v.x * v.x + v.y * v.y;
        } else if (OUT == 2) {
            const float r = v.x * v.x + v.y * v.y - __ldg(aux + o);
            lsum = fmaf(r, r, lsum);
            static_cast<float2*>(dst)[o] = make_float2(4.f * r * v.x, 4.f * r * v.y);
        } else {
            const float ph = __ldg(aux + o) * s;
            const float at = expf(-ph * ib);
            float sn, cs;
            sincosf(ph, &sn, &cs);
            const float px = at * cs, py = at * sn;             // psi
            const float wx = -ib * px - py, wy = px - ib * py;  // (i - ib) psi
            static_cast<float*>(dst)[o] = s * (v.x * wx + v.y * wy);
        }
    };
    stockham::pairconv<N>(sm, ad, ld, pair, st, g, tw, tw + 3 * N / 2);
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
}

// ---------------------------------------------------------------- general sizes
// v[t][p][q] = a[t][sig(p)][sig(q)] (IN 0: complex a; IN 1: a = psi(p s)).
template <int IN>
__global__ void k_gen_load(const void* __restrict__ src, float2* __restrict__ v, long total, int nz, int n, float s,
                           float ib) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int q = (int)(i % n);
        const long r = i / n;
        const int p = (int)(r % nz);
        const long t = r / nz;
        const long o = (t * nz + sig(p, nz)) * n + sig(q, n);
        if (IN == 0) {
            v[i] = __ldg(static_cast<const float2*>(src) + o);
        } else {
            const float ph = __ldg(static_cast<const float*>(src) + o) * s;
            const float at = expf(-ph * ib);
            float sn, cs;
            sincosf(ph, &sn, &cs);
            v[i] = make_float2(at * cs, at * sn);
        }
    }
}

// W[k][l] = sum over the four reflections of V (y and x pair tables).
__global__ void k_gen_mix(const float2* __restrict__ V, float2* __restrict__ W, const float4* __restrict__ Sy,
                          const float4* __restrict__ Sx, long total, int nz, int n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        const int l = (int)(i % n);
        const long r = i / n;
        const int k = (int)(r % nz);
        const float2* fr = V + (r / nz) * nz * n;
        const int kr = k == 0 ? 0 : nz - k, lr = l == 0 ? 0 : n - l;
        const float4 y = __ldg(Sy + k), x = __ldg(Sx + l);
        const float2 py = make_float2(y.x, y.y), qy = make_float2(y.z, y.w);
        const float2 px = make_float2(x.x, x.y), qx = make_float2(x.z, x.w);
        const float2 a = cmul(__ldg(fr + (long)k * n + l), px);
        const float2 b = cmul(__ldg(fr + (long)k * n + lr), qx);
        const float2 c = cmul(__ldg(fr + (long)kr * n + l), px);
        const float2 d = cmul(__ldg(fr + (long)kr * n + lr), qx);
        const float2 ab = cmul(make_float2(a.x + b.x, a.y + b.y), py);
        const float2 cd = cmul(make_float2(c.x + d.x, c.y + d.y), qy);
        W[i] = make_float2(ab.x + cd.x, ab.y + cd.y);
    }
}

// out[t][sig(p)][sig(q)] from w[t][p][q]; one block per (t, p) row.  OUT as
// in k_xpass; OUT 2 writes one partial per row.
template <int OUT>
__global__ void k_gen_store(const float2* __restrict__ w, void* __restrict__ dst, int nz, int n,
                            const float* __restrict__ aux, float* __restrict__ partials, float s, float ib) {
    __shared__ float red[32];
    const long row = blockIdx.x;  // t * nz + p
    const int p = (int)(row % nz);
    const long orow = (row - p + sig(p, nz)) * n;
    float lsum = 0.f;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const float2 v = w[row * n + q];
        const long o = orow + sig(q, n);
        if (OUT == 0) {
            static_cast<float2*>(dst)[o] = v;
        } else if (OUT == 1) {
            static_cast<float*>(dst)[o] = v.x * v.x + v.y * v.y;
        } else if (OUT == 2) {
            const float r = v.x * v.x + v.y * v.y - __ldg(aux + o);
            lsum = fmaf(r, r, lsum);
            static_cast<float2*>(dst)[o] = make_float2(4.f * r * v.x, 4.f * r * v.y);
        } else {
            const float ph = __ldg(aux + o) * s;
            const float at = expf(-ph * ib);
            float sn, cs;
            sincosf(ph, &sn, &cs);
            const float px = at * cs, py = at * sn;
            const float wx = -ib * px - py, wy = px - ib * py;
            static_cast<float*>(dst)[o] = s * (v.x * wx + v.y * wy);
        }
    }
    if (OUT == 2) {
        for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            float t = 0.f;
            for (int i = 0; i < (int)(blockDim.x + 31) / 32; ++i) t += red[i];
            partials[row] = t;
        }
    }
}

// ---------------------------------------------------------------- launch
template <int N>
constexpr int y_cols() {
    constexpr int G = stockham::Sched<N>::G;
    return 256 / G < 4 ? 4 : (256 / G > 32 ? 32 : 256 / G);
}
template <int N>
constexpr int x_rows() {
    constexpr int G = stockham::Sched<N>::G;
    return G >= 256 ? 1 : 256 / G;
}

template <int N, int IN>
int launch_y(mm_prop* h, const void* src, int ntheta, const float4* S, float s, float ib, cudaStream_t st) {
    constexpr int G = stockham::Sched<N>::G;
    constexpr int CW = y_cols<N>();
    const size_t smem = (size_t)stockham::ColAddr<CW>::rows(N) * CW * sizeof(float2);
    if constexpr (stockham::Sched<N>::P2 && N >= 64 && N <= 1024) {
        constexpr int CWp = pf_cols<N>();
        if (h->n % CWp == 0) {  // persistent prefetching column pass
            const size_t smem = (size_t)stockham::ColAddr<CWp>::rows(N) * CWp * sizeof(float2);
            auto kern = h->n == 2048 ? k_ypass_pf<N, IN, 2048> : k_ypass_pf<N, IN, 0>;
            MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            int dev = 0, sms = 0, per_sm = 0;
            MM_CUDA(cudaGetDevice(&dev));
            MM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            MM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CWp * G, smem));
            const long items = (long)ntheta * (h->n / CWp);
            const long blocks = std::min<long>(items, (long)sms * std::max(per_sm, 1));
            h->tm.begin(0, st);
            kern<<<(unsigned)blocks, dim3(CWp, G), smem, st>>>(src, h->mid, S, h->twy, items, h->n, s, ib);
            MM_LAUNCHED();
            h->tm.end(st, 1);
            return MM_OK;
        }
    }
    auto kern = h->n == 2048 ? k_ypass<N, CW, IN, 2048> : k_ypass<N, CW, IN, 0>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // one frame per grid row: frames go in launches of at most 65535 (the grid's y limit)
    const size_t esz = IN == 0 ? sizeof(float2) : sizeof(float);
    const long frame = (long)N * h->n;
    int launches = 0;
    h->tm.begin(0, st);
    for (int t0 = 0; t0 < ntheta; t0 += 65535) {
        const int nt = ntheta - t0 < 65535 ? ntheta - t0 : 65535;
        dim3 block(CW, G), grid((h->n + CW - 1) / CW, nt);
        kern<<<grid, block, smem, st>>>(static_cast<const char*>(src) + (size_t)t0 * frame * esz,
                                        h->mid + (size_t)t0 * frame, S, h->twy, h->n, s, ib);
        MM_LAUNCHED();
        ++launches;
    }
    h->tm.end(st, launches);
    return MM_OK;
}

template <int N, int OUT>
int launch_x(mm_prop* h, void* dst, int ntheta, const float4* S, cudaStream_t st, const float* aux = nullptr,
             float* partials = nullptr, float s = 0.f, float ib = 0.f) {
    constexpr int G = stockham::Sched<N>::G;
    constexpr int RPB = x_rows<N>();
    const size_t smem = (size_t)RPB * (N + N / 16) * sizeof(float2);
    auto kern = k_xpass<N, RPB, OUT>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const long rows = (long)ntheta * h->nz;
    dim3 block(G, RPB), grid((unsigned)((rows + RPB - 1) / RPB));
    h->tm.begin(1, st);
    kern<<<grid, block, smem, st>>>(h->mid, dst, S, h->twx, rows, aux, partials, s, ib);
    MM_LAUNCHED();
    h->tm.end(st, 1);
    return MM_OK;
}

// Column pass of distance j; adj selects the conj(K) tables.
// Line lengths with native kernels: powers of two in [2, 2048] and
// 3 * 2^k in [96, 3072]; other sizes take the cuFFT path.
bool native_len(int L) {
    return mm_is_pow2(L) ? (L >= 2 && L <= 2048) : (stockham::length_ok(L) && L >= 96 && L <= 3072);
}

template <int IN>
int dispatch_y(mm_prop* h, const void* src, int ntheta, int j, bool adj, float s, float ib, cudaStream_t st) {
    const float4* S = h->Sy + ((size_t)j * 2 + (adj ? 1 : 0)) * h->nz;
    switch (h->nz) {
        case 2: return launch_y<2, IN>(h, src, ntheta, S, s, ib, st);
        case 4: return launch_y<4, IN>(h, src, ntheta, S, s, ib, st);
        case 8: return launch_y<8, IN>(h, src, ntheta, S, s, ib, st);
        case 16: return launch_y<16, IN>(h, src, ntheta, S, s, ib, st);
        case 32: return launch_y<32, IN>(h, src, ntheta, S, s, ib, st);
        case 64: return launch_y<64, IN>(h, src, ntheta, S, s, ib, st);
        case 128: return launch_y<128, IN>(h, src, ntheta, S, s, ib, st);
        case 256: return launch_y<256, IN>(h, src, ntheta, S, s, ib, st);
        case 512: return launch_y<512, IN>(h, src, ntheta, S, s, ib, st);
        case 1024: return launch_y<1024, IN>(h, src, ntheta, S, s, ib, st);
        case 2048: return launch_y<2048, IN>(h, src, ntheta, S, s, ib, st);
        case 96: return launch_y<96, IN>(h, src, ntheta, S, s, ib, st);
        case 192: return launch_y<192, IN>(h, src, ntheta, S, s, ib, st);
        case 384: return launch_y<384, IN>(h, src, ntheta, S, s, ib, st);
        case 768: return launch_y<768, IN>(h, src, ntheta, S, s, ib, st);
        case 1536: return launch_y<1536, IN>(h, src, ntheta, S, s, ib, st);
        case 3072: return launch_y<3072, IN>(h, src, ntheta, S, s, ib, st);
    }
    MM_REQUIRE(false, "unsupported nz=%d", h->nz);
}

template <int OUT>
int dispatch_x(mm_prop* h, void* dst, int ntheta, int j, bool adj, cudaStream_t st, const float* aux = nullptr,
               float* partials = nullptr, float s = 0.f, float ib = 0.f) {
    const float4* S = h->Sx + ((size_t)j * 2 + (adj ? 1 : 0)) * h->n;
    switch (h->n) {
        case 2: return launch_x<2, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 4: return launch_x<4, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 8: return launch_x<8, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 16: return launch_x<16, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 32: return launch_x<32, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 64: return launch_x<64, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 128: return launch_x<128, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 256: return launch_x<256, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 512: return launch_x<512, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 1024: return launch_x<1024, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 2048: return launch_x<2048, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 96: return launch_x<96, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 192: return launch_x<192, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 384: return launch_x<384, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 768: return launch_x<768, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 1536: return launch_x<1536, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
        case 3072: return launch_x<3072, OUT>(h, dst, ntheta, S, st, aux, partials, s, ib);
    }
    MM_REQUIRE(false, "unsupported n=%d", h->n);
}

// cuFFT 2-D plan over `nt` frames of nz x n (cached: all frames, and the last
// smaller batch).
int gen_plan(mm_prop* h, int nt, cufftHandle* out) {
    cufftHandle* slot = nt == h->ntheta ? &h->plan_full : &h->plan_part;
    if (nt != h->ntheta && h->part_batch != nt && h->plan_part) {
        cufftDestroy(h->plan_part);
        h->plan_part = 0;
    }
    if (!*slot) {
        // 64-bit plan: a batch of frames of the largest sizes (24576^2 and up)
        // holds more than 2^31 elements
        long long dims[2] = {h->nz, h->n};
        size_t ws = 0;
        MM_CUFFT(cufftCreate(slot));
        const cufftResult r = cufftMakePlanMany64(*slot, 2, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2C, nt, &ws);
        if (r != CUFFT_SUCCESS) {
            cufftDestroy(*slot);
            *slot = 0;
            mm::set_error("cufftMakePlanMany64 (%d frames of %d x %d): %s", nt, h->nz, h->n, mm::cufft_name(r));
            return MM_ECUFFT;
        }
        if (nt != h->ntheta) h->part_batch = nt;
    }
    *out = *slot;
    return MM_OK;
}

// One D (adj = false) or DT (adj = true) on general sizes: IN / OUT as in
// the fused passes.
template <int IN, int OUT>
int run_general(mm_prop* h, const void* src, void* dst, int nt, int j, bool adj, cudaStream_t st,
                const float* aux = nullptr, float* partials = nullptr, float s = 0.f, float ib = 0.f) {
    const long total = (long)nt * h->nz * h->n;
    const int bs = 256;
    const unsigned grid = (unsigned)std::min<long>((total + bs - 1) / bs, 148L * 16);
    cufftHandle plan;
    MM_TRY(gen_plan(h, nt, &plan));
    MM_CUFFT(cufftSetStream(plan, st));
    h->tm.begin(0, st);
    k_gen_load<IN><<<grid, bs, 0, st>>>(src, h->mid, total, h->nz, h->n, s, ib);
    MM_LAUNCHED();
    MM_CUFFT(cufftExecC2C(plan, (cufftComplex*)h->mid, (cufftComplex*)h->mid2, CUFFT_FORWARD));
    const float4* Sy = h->Sy + ((size_t)j * 2 + (adj ? 1 : 0)) * h->nz;
    const float4* Sx = h->Sx + ((size_t)j * 2 + (adj ? 1 : 0)) * h->n;
    k_gen_mix<<<grid, bs, 0, st>>>(h->mid2, h->mid, Sy, Sx, total, h->nz, h->n);
    MM_LAUNCHED();
    MM_CUFFT(cufftExecC2C(plan, (cufftComplex*)h->mid, (cufftComplex*)h->mid2, CUFFT_INVERSE));
    h->tm.end(st, 2);
    h->tm.begin(1, st);
    k_gen_store<OUT><<<(unsigned)((long)nt * h->nz), 256, 0, st>>>(h->mid2, dst, h->nz, h->n, aux, partials, s, ib);
    MM_LAUNCHED();
    h->tm.end(st, 1);
    return MM_OK;
}

// asz / bsz: bytes per pixel of the input a and the output b (range checks).
int check_call(const mm_prop* h, const void* a, const void* b, int ntheta, int j, const char* who, int asz = 8,
               int bsz = 8) {
    MM_REQUIRE(h != nullptr, "%s: NULL handle", who);
    MM_REQUIRE(a != nullptr && b != nullptr, "%s: NULL array", who);
    MM_REQUIRE(ntheta >= 1 && ntheta <= h->ntheta, "%s: ntheta=%d outside [1, %d]", who, ntheta, h->ntheta);
    MM_REQUIRE(j >= 0 && j < h->ndist, "%s: distance index %d outside [0, %d)", who, j, h->ndist);
    const size_t px = (size_t)ntheta * h->nz * h->n;
    MM_RANGE(a, px * asz, who, "input");
    MM_RANGE(b, px * bsz, who, "output");
    return MM_OK;
}

void destroy(mm_prop* h) {
    h->tm.release();
    if (h->plan_full) cufftDestroy(h->plan_full);
    if (h->plan_part) cufftDestroy(h->plan_part);
    void* bufs[] = {h->Sx, h->Sy, h->twx, h->twy, h->mid, h->mid2};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete h;
}

// P/Q entry k of an N-point line (see the top of this file) for distance z:
// the chirp exp(-i pi lambda z f^2) / (2N) on the float32 fftfreq grid of the
// 2N padded points (processing/propagation.py:23-31), phases in FP64 reduced
// mod 2 pi.  Host and device (allocation-free path) share this code.
__host__ __device__ inline void chirp_2n(int k, int N, double voxelsize, double wavelength, double z, double* re,
                                          double* im) {
    const int L = 2 * N;
    const double val = 1.0 / (L * voxelsize);
    const int kk = k < (L + 1) / 2 ? k : k - L;
    const double f = (double)(float)(kk * val);
    const double ph = fmod(M_PI * wavelength * z * f * f, 2.0 * M_PI);
    *re = cos(-ph) / L;
    *im = sin(-ph) / L;
}
__host__ __device__ inline float4 pq_entry(int k, int N, double voxelsize, double wavelength, double z, bool adj) {
    double ar, ai, br, bi;
    chirp_2n(k, N, voxelsize, wavelength, z, &ar, &ai);
    chirp_2n(k == 0 ? 0 : N - k, N, voxelsize, wavelength, z, &br, &bi);
    if (adj) {
        ai = -ai;
        bi = -bi;
    }
    const double pr = ar + br, pi = ai + bi, dr = ar - br, di = ai - bi;
    const double c = cos(M_PI * k / N), s = sin(M_PI * k / N);
    const double qr = k == 0 ? 0.0 : c * dr - s * di, qi = k == 0 ? 0.0 : c * di + s * dr;
    return make_float4((float)pr, (float)pi, (float)qr, (float)qi);
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
    MM_REQUIRE(n >= 2 && n <= 32768 && nz >= 2 && nz <= 32768, "mm_prop_create: n=%d, nz=%d outside [2, 32768]", n,
               nz);
    MM_REQUIRE(ntheta >= 1 && ndist >= 1 && distance_host != nullptr, "mm_prop_create: bad ntheta/ndist");
    MM_REQUIRE(voxelsize > 0, "mm_prop_create: voxelsize must be positive");
    MM_CUDA(mmfft::init_constants());
    mm_prop* h = new mm_prop();
    h->n = n;
    h->nz = nz;
    h->ntheta = ntheta;
    h->ndist = ndist;
    h->general = !(native_len(n) && native_len(nz));
    std::vector<float4> sx((size_t)ndist * 2 * n), sy((size_t)ndist * 2 * nz);
    std::vector<float2> tx, ty;
    for (int j = 0; j < ndist; ++j)
        for (int a = 0; a < 2; ++a) {
            for (int k = 0; k < n; ++k)
                sx[((size_t)j * 2 + a) * n + k] = pq_entry(k, n, voxelsize, wavelength, distance_host[j], a == 1);
            for (int k = 0; k < nz; ++k)
                sy[((size_t)j * 2 + a) * nz + k] = pq_entry(k, nz, voxelsize, wavelength, distance_host[j], a == 1);
        }
    if (!h->general) {
        twiddles(tx, n);
        twiddles(ty, nz);
    }
    struct B { void** p; const void* v; size_t bytes; const char* what; } bs[] = {
        {(void**)&h->Sx, sx.data(), sx.size() * sizeof(float4), "x line tables"},
        {(void**)&h->Sy, sy.data(), sy.size() * sizeof(float4), "y line tables"},
        {(void**)&h->twx, tx.data(), tx.size() * sizeof(float2), "x twiddles"},
        {(void**)&h->twy, ty.data(), ty.size() * sizeof(float2), "y twiddles"}};
    for (auto& b : bs) {
        if (b.bytes == 0) continue;
        int rc = dev_alloc(b.p, b.bytes, b.what);
        if (rc != MM_OK) {
            destroy(h);
            return rc;
        }
        h->ws_bytes += b.bytes;
        if (cudaMemcpy(*b.p, b.v, b.bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            mm::set_error("mm_prop_create: table upload failed");
            destroy(h);
            return MM_ECUDA;
        }
    }
    const size_t mid = (size_t)ntheta * nz * n;
    int rc = dev_alloc((void**)&h->mid, mid * sizeof(float2), "propagator intermediate");
    if (rc == MM_OK && h->general) rc = dev_alloc((void**)&h->mid2, mid * sizeof(float2), "propagator spectrum");
    if (rc != MM_OK) {
        destroy(h);
        return rc;
    }
    h->ws_bytes += mid * sizeof(float2) * (h->general ? 2 : 1);
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
    if (h->general) return run_general<0, 0>(h, psi, out, ntheta, j, false, st);
    MM_TRY((dispatch_y<0>(h, psi, ntheta, j, false, 0.f, 0.f, st)));
    return dispatch_x<0>(h, out, ntheta, j, false, st);
}

extern "C" int mm_prop_DT(mm_prop* h, const void* g, void* out, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, g, out, ntheta, j, "mm_prop_DT"));
    cudaStream_t st = (cudaStream_t)stream;
    if (h->general) return run_general<0, 0>(h, g, out, ntheta, j, true, st);
    MM_TRY((dispatch_y<0>(h, g, ntheta, j, true, 0.f, 0.f, st)));
    return dispatch_x<0>(h, out, ntheta, j, true, st);
}

extern "C" int mm_prop_intensity(mm_prop* h, const float* proj, float inv_norm, float inv_beta_ratio,
                                 float* intensity, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, proj, intensity, ntheta, j, "mm_prop_intensity", 4, 4));
    cudaStream_t st = (cudaStream_t)stream;
    if (h->general)
        return run_general<1, 1>(h, proj, intensity, ntheta, j, false, st, nullptr, nullptr, inv_norm, inv_beta_ratio);
    MM_TRY((dispatch_y<1>(h, proj, ntheta, j, false, inv_norm, inv_beta_ratio, st)));
    return dispatch_x<1>(h, intensity, ntheta, j, false, st);
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
// column-pass intermediate -- lives in the file-scope array below.  CUDA
// loads a library's device code lazily by default (CUDA_MODULE_LOADING=LAZY
// since 12.2), so a GPU takes the array's kNoAllocBytes when this file's
// device code is first loaded there -- at the latest in the first call's
// cudaGetSymbolAddress -- and keeps them until the process exits.  A caller
// that reserves its device memory pool up front must therefore make one call
// (any valid size) on each device before reserving the pool, and before any
// stream capture.  All calls share that one array and it keeps the last
// call's contents, so calls that overlap on the GPU (two streams, two host
// threads) race; callers must order them.  Nothing in it needs to start at
// zero: every call rewrites the tables and the intermediate before reading
// them.
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

// Line and twiddle tables of one distance, computed on the device in FP64
// exactly as pq_entry() / twiddles() do on the host for mm_prop_create.
__global__ void k_noalloc_tables(float4* __restrict__ Sx, float4* __restrict__ Sy, float2* __restrict__ twx,
                                 float2* __restrict__ twy, int n, int nz, double wavelength, double voxelsize,
                                 double z) {
    const int total = n + nz + 3 * n + 3 * nz;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        int i = t;
        if (i < n + nz) {  // P/Q along x then y
            const bool along_x = i < n;
            const int N = along_x ? n : nz;
            const int k = along_x ? i : i - n;
            const float4 e = pq_entry(k, N, voxelsize, wavelength, z, false);
            if (along_x) Sx[k] = e; else Sy[k] = e;
            continue;
        }
        i -= n + nz;  // twiddles: x slot (3n) then y slot (3nz)
        const bool along_x = i < 3 * n;
        const int len = along_x ? n : nz;
        int q = along_x ? i : i - 3 * n;
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
    MM_REQUIRE(mm_is_pow2(n) && n >= 2 && n <= 2048, "mm_prop_D_noalloc: n=%d must be a power of two in [2, 2048]",
               n);
    MM_REQUIRE(mm_is_pow2(nz) && nz >= 2 && nz <= 2048,
               "mm_prop_D_noalloc: nz=%d must be a power of two in [2, 2048]", nz);
    MM_REQUIRE(ntheta >= 1 && voxelsize > 0, "mm_prop_D_noalloc: bad ntheta/voxelsize");
    const size_t tables = (size_t)8 * n + 8 * nz;
    const size_t need = (tables + (size_t)ntheta * nz * n) * sizeof(float2);
    MM_REQUIRE(need <= kNoAllocBytes,
               "mm_prop_D_noalloc: ntheta*nz*n=%zu needs %zu bytes of scratch, more than the %zu-byte "
               "static buffer (use mm_prop_D, or fewer angles per call)",
               (size_t)ntheta * nz * n, need, kNoAllocBytes);
    MM_RANGE(psi, (size_t)ntheta * nz * n * 8, "mm_prop_D_noalloc", "psi");
    MM_RANGE(out, (size_t)ntheta * nz * n * 8, "mm_prop_D_noalloc", "out");
    float2* base = nullptr;
    MM_TRY(noalloc_setup(&base));
    cudaStream_t st = (cudaStream_t)stream;
    mm_prop h;  // view onto the static scratch; owns nothing
    h.n = n;
    h.nz = nz;
    h.ntheta = ntheta;
    h.ndist = 1;
    // float2 slots: Sx (n float4) | Sy (nz float4) | twx (3n) | twy (3nz) | ... | mid at 8(n + nz)
    h.Sx = reinterpret_cast<float4*>(base);
    h.Sy = reinterpret_cast<float4*>(base + 2 * n);
    h.twx = base + 2 * n + 2 * nz;
    h.twy = h.twx + 3 * n;
    h.mid = base + tables;
    k_noalloc_tables<<<(unsigned)((tables + 255) / 256), 256, 0, st>>>(h.Sx, h.Sy, h.twx, h.twy, n, nz, wavelength,
                                                                      voxelsize, distance);
    MM_LAUNCHED();
    MM_TRY((dispatch_y<0>(&h, psi, ntheta, 0, false, 0.f, 0.f, st)));
    return dispatch_x<0>(&h, out, ntheta, 0, false, st);
}

extern "C" long mm_prop_grad_partials(mm_prop* h, int ntheta) {
    if (!h || ntheta < 1) return 0;
    if (h->general) return (long)ntheta * h->nz;
    // threads per row line of the x-pass (stockham::Sched<n>::G): 16 values
    // per thread for 2^k, 24 for 3 * 2^k; rows per block as x_rows()
    const bool p2 = mm_is_pow2(h->n);
    const int V = p2 ? 16 : 24;
    const int G = h->n >= V ? h->n / V : 1;
    const int rpb = G >= 256 ? 1 : 256 / G;
    return ((long)ntheta * h->nz + rpb - 1) / rpb;
}

extern "C" int mm_prop_grad_forward(mm_prop* h, const float* proj, const float* data, float inv_norm,
                                    float inv_beta_ratio, void* gu, float* partials, int ntheta, int j,
                                    void* stream) {
    MM_TRY(check_call(h, proj, gu, ntheta, j, "mm_prop_grad_forward", 4, 8));
    MM_REQUIRE(data != nullptr && partials != nullptr, "mm_prop_grad_forward: NULL data/partials");
    MM_RANGE(data, (size_t)ntheta * h->nz * h->n * 4, "mm_prop_grad_forward", "data");
    MM_RANGE(partials, (size_t)mm_prop_grad_partials(h, ntheta) * 4, "mm_prop_grad_forward", "partials");
    cudaStream_t st = (cudaStream_t)stream;
    if (h->general)
        return run_general<1, 2>(h, proj, gu, ntheta, j, false, st, data, partials, inv_norm, inv_beta_ratio);
    MM_TRY((dispatch_y<1>(h, proj, ntheta, j, false, inv_norm, inv_beta_ratio, st)));
    return dispatch_x<2>(h, gu, ntheta, j, false, st, data, partials, inv_norm, inv_beta_ratio);
}

extern "C" int mm_prop_grad_backward(mm_prop* h, const void* gu, const float* proj, float inv_norm,
                                     float inv_beta_ratio, float* gp, int ntheta, int j, void* stream) {
    MM_TRY(check_call(h, gu, gp, ntheta, j, "mm_prop_grad_backward", 8, 4));
    MM_REQUIRE(proj != nullptr, "mm_prop_grad_backward: NULL proj");
    MM_RANGE(proj, (size_t)ntheta * h->nz * h->n * 4, "mm_prop_grad_backward", "proj");
    cudaStream_t st = (cudaStream_t)stream;
    if (h->general)
        return run_general<0, 3>(h, gu, gp, ntheta, j, true, st, proj, nullptr, inv_norm, inv_beta_ratio);
    MM_TRY((dispatch_y<0>(h, gu, ntheta, j, true, 0.f, 0.f, st)));
    return dispatch_x<3>(h, gp, ntheta, j, true, st, proj, nullptr, inv_norm, inv_beta_ratio);
}
