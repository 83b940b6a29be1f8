// Internals shared by the translation units of the USFFT Radon pair
// (tomo.cu: handle, forward, x/r-side transforms, gather; tomo_scatter.cu:
// the adjoint's scatter table and scatter kernels).
#pragma once

#include "mm_common.cuh"
#include "fft_smem.cuh"

#include <cuda_bf16.h>
#include <cufft.h>

#include <vector>

// The adjoint's static scatter table for the angles [t0, t1): destination
// cell pair (row, 2p), (row, 2p+1) -> entries (sample, conj bits) + weights.
struct ScatterTable {
    int t0 = 0, t1 = 0;
    unsigned* ptr = nullptr;      // npairs + 1
    unsigned* idx = nullptr;      // sample index (k*T + t) | conj left << 31 | conj right << 30
    float2* w = nullptr;          // (left, right) weights
    // pairs whose lists exceed kChunk entries (the cells around the spectrum
    // origin collect thousands) are summed in kChunk-entry pieces by separate
    // warps and combined in piece order
    uint2* chunk_task = nullptr;  // (first, end) entry of each piece
    uint4* chunk_pair = nullptr;  // (pair, first piece, end piece, 0) per long pair
    float2* chunk_part = nullptr; // (pieces, 2, zs) partial sums: left and right cell
    long nchunks = 0, nlong = 0, nnz = 0;
    size_t bytes = 0;
};

struct mm_tomo {
    int n = 0, nz = 0, ntheta = 0, m = 0, zs = 0, K = 0, clamp = 0, compensated = 0;
    int paired = 0;  // angles symmetric under theta -> theta + pi: the gather takes them in pairs
    float mu = 0.f, c0 = 0.f, c1 = 0.f, phi_scale = 0.f;
    int device = 0;
    float* d_cos = nullptr;
    float* d_sin = nullptr;
    float* d_phi1 = nullptr;
    float2* d_twy = nullptr;     // Stockham twiddles of the 2n-point x and column transforms
    float2* d_tww = nullptr;     // the same for the wide 3 * 2^k schedule (2n >= 6144)
    float2* d_twr = nullptr;     // Stockham twiddles of the n/2-point r transforms
    float2* d_exr = nullptr;     // e^{+2 pi i k/n}, k = 0..n/2 (real-from-half-length packing)
    float2* col_scratch = nullptr;  // L2-resident per-SM regions of the 64 x 64 column transform
    float2* col_tw = nullptr;       // its W_4096^(n2 k1) table
    int sms = 0;
    bool fused_x = false, fused_r = false;
    // forward buffers
    float* P = nullptr;          // (zs, n, 2n)     padded phi*obj rows
    float2* X = nullptr;         // (zs, n, n+1)    row spectra
    float2* Y = nullptr;         // (2n, n+1, zs)   row spectra in centre rows, zero elsewhere
    float2* F = nullptr;         // (2n, n+1, zs)   half spectrum, raw fftfreq order
    float2* Hh = nullptr;        // (n/2+1, T, zs)  C2R input along r
    float* sino_tmp = nullptr;   // (T, zs, n)      only when nz < zs
    void* fft_work = nullptr;
    size_t fft_work_bytes = 0;
    cufftHandle plan_xr2c = 0, plan_xc2r = 0, plan_y = 0, plan_rc2r = 0, plan_rr2c = 0, plan_rc2c = 0;
    bool plans_rt = false, plans_c = false;
    bool y_dirty = false;        // RT used Y as scratch: its zero pad rows need restoring
    // adjoint scatter table
    // adjoint scatter tables, one per block of angles (the scatter of every
    // block after the first adds into the first one's result)
    bool csr_ready = false;
    bool tables_resident = true;  // false: rebuilt block by block at every RT call
    int table_angles = 0;         // angles per table block
    std::vector<ScatterTable> tabs;
    float* ypad = nullptr;       // (T, zs, n) real sino padded in z (nz < zs)
    float2* yc = nullptr;        // (T, zs, n) complex sino spectrum (complex RT)
    size_t ws_bytes = 0;
    mm::StageTimer tm;
};

namespace {

constexpr int kThreads = 256;

// --------------------------------------------------------------------------
// Sample geometry shared by the gather and the scatter-table builder.
// Coordinates follow processing/kernels.py:293-299 in float32; cos/sin come
// from an FP64 table.  Samples with x0 < 0 are taken at -p (Hermitian).
struct SampleGeo {
    int j, bx, by;
    bool mir;
    float x0, y0;
};

__device__ __forceinline__ SampleGeo sample_geo(int t, int k, int n, int M, const float* __restrict__ cosT,
                                                const float* __restrict__ sinT, bool clamp = false) {
    SampleGeo g;
    g.j = (k < n / 2) ? k + n / 2 : 0;
    const float cx = n * 0.5f;
    const float r = ((float)g.j - cx) / (float)n;
    float x0 = r * __ldg(cosT + t);
    float y0 = -r * __ldg(sinT + t);
    if (clamp) {  // TomoLargeReal's gather (processing/kernels.py:478-481)
        x0 = fminf(fmaxf(x0, -0.5f), 0.5f - 1e-5f);
        y0 = fminf(fmaxf(y0, -0.5f), 0.5f - 1e-5f);
    }
    g.mir = x0 < 0.f;
    if (g.mir) {
        x0 = -x0;
        y0 = -y0;
    }
    const float ftwon = (float)(2 * n);
    g.bx = __float2int_rn(ftwon * x0) - M;   // rintf: round half to even
    g.by = __float2int_rn(ftwon * y0) - M;
    g.x0 = x0;
    g.y0 = y0;
    return g;
}

// Gaussian weight of tap offset i along one axis; `sgn` folds the
// (-1)^(k0+k1) shift of processing/kernels.py:319-321 in per axis.
__device__ __forceinline__ float tap_weight(int ell, float pos, float inv_twon, float c1) {
    const float w = (float)ell * inv_twon - pos;
    const float e = expf(c1 * w * w);
    return (ell & 1) ? -e : e;
}

// Weights of one or two samples spread over a warp whose 32 lanes all work on
// the same sample(s): lane q computes weight q (and q + 32) of the list
// (wx of a, wy of a, wx of b, wy of b), each 2m+1 long, and every lane reads
// the list back by shuffles -- the same float values as each lane computing
// all of them, at one or two exponentials per lane instead of 4(2m+1).
template <int L, int NS>
struct WarpWeights {
    float w0, w1;
    __device__ __forceinline__ static float one(int q, const SampleGeo& ga, const SampleGeo& gb, float inv_twon,
                                                float c0, float c1) {
        const int which = q / L, i = q - which * L;
        const bool b = which >= 2, y = which & 1;
        const int base = b ? (y ? gb.by : gb.bx) : (y ? ga.by : ga.bx);
        const float pos = b ? (y ? gb.y0 : gb.x0) : (y ? ga.y0 : ga.x0);
        const float v = tap_weight(base + i, pos, inv_twon, c1);
        return y ? c0 * v : v;
    }
    __device__ __forceinline__ WarpWeights(int lane, const SampleGeo& ga, const SampleGeo& gb, float inv_twon,
                                           float c0, float c1) {
        constexpr int NW = 2 * NS * L;
        static_assert(NW <= 64, "weights of at most two rounds of 32 lanes");
        w0 = one(min(lane, NW - 1), ga, gb, inv_twon, c0, c1);
        w1 = NW > 32 ? one(min(lane + 32, NW - 1), ga, gb, inv_twon, c0, c1) : 0.f;
    }
    // weight q of the list (q a compile-time index after unrolling)
    __device__ __forceinline__ float get(int q) const {
        return q < 32 ? __shfl_sync(0xffffffffu, w0, q) : __shfl_sync(0xffffffffu, w1, q - 32);
    }
};

// Destination of tap (u, v) in the stored half plane (columns 0..n, rows in
// raw order): reflected through the origin when u is outside [0, n].
__device__ __forceinline__ void tap_cell(int u, int v, int n, int& row, int& col, bool& cj) {
    const int twon = 2 * n;
    if (u >= 0 && u <= n) {
        col = u;
        cj = false;
    } else {
        col = (u < 0) ? -u : twon - u;
        v = -v;
        cj = true;
    }
    row = v < 0 ? v + twon : (v >= twon ? v - twon : v);
}

// float32 or bfloat16 storage of the volume and the sinogram; arithmetic is
// float32 either way.
__device__ __forceinline__ float ld_elem(const float* p) { return __ldg(p); }
__device__ __forceinline__ float ld_elem(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ void st_elem(float* p, float v) { *p = v; }
__device__ __forceinline__ void st_elem(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ float2 ld_pair(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ float2 ld_pair(const __nv_bfloat16* p) {
    return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(p));
}
__device__ __forceinline__ void st_pair(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }
__device__ __forceinline__ void st_pair(__nv_bfloat16* p, float2 v) {
    *reinterpret_cast<__nv_bfloat162*>(p) = __float22bfloat162_rn(v);
}

template <int ZV>
struct ZVec;
template <>
struct ZVec<1> {
    static __device__ __forceinline__ void load(const float2* p, float* v) {
        float2 a = __ldg(p);
        v[0] = a.x; v[1] = a.y;
    }
    static __device__ __forceinline__ void store(float2* p, const float* v) {
        *p = make_float2(v[0], v[1]);
    }
};
template <>
struct ZVec<2> {
    static __device__ __forceinline__ void load(const float2* p, float* v) {
        float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    static __device__ __forceinline__ void store(float2* p, const float* v) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
};

template <typename Tp>
int alloc(mm_tomo* h, Tp** p, size_t count, const char* what) {
    void* q = nullptr;
    MM_TRY(mm::dev_alloc(&q, count * sizeof(Tp), what));
    *p = static_cast<Tp*>(q);
    h->ws_bytes += count * sizeof(Tp);
    return MM_OK;
}

// Padded line lengths 2n with native shared-memory column transforms:
// powers of two in [16, 4096] and 3 * 2^k in [96, 6144].
inline bool native_line(long L) {
    return stockham::length_ok(L) && (mm_is_pow2(L) ? (L >= 16 && L <= 4096) : (L >= 96 && L <= 6144));
}

int pick_lanes(int zs, int& ZV, int& LPS) {
    if (zs >= 64) { ZV = 2; LPS = 32; }
    else if (zs >= 2) { ZV = 2; LPS = zs / 2; }
    else { ZV = 1; LPS = 1; }
    return MM_OK;
}

}  // namespace

namespace mmtomo {
// tomo_scatter.cu
int build_csr(mm_tomo* h, cudaStream_t st);
void free_tables(mm_tomo* h);
int launch_scatter(mm_tomo* h, const float2* Q, float2* A, cudaStream_t st);
}  // namespace mmtomo
