// USFFT Radon pair (TomoReal / TomoLargeReal .R and .RT) for sm_100a.
//
// Reference operator (processing/tomo.py:121-188, processing/kernels.py):
//   R(obj)  = Re( c . IFFT_r( c . (1/n) G F2( pad2n(phi . obj) ) ) ) / 4
//   RT(y)   = phi . crop( c2 . IFFT2( c2 . G^H( c . FFT_r(c . y) ) ) )
// with G the (2m+1)^2 Gaussian gather onto the polar grid.
//
// B200 formulation (same operator, different schedule and layout):
//  * Slices are interleaved in the spectrum: F[v][u][z] with z innermost, so
//    one warp owns one polar sample for 32..64 slices; the Gaussian weights
//    are computed once per sample and every tap is one coalesced 256/512-byte
//    load.
//  * Real input makes the spectrum and every polar line Hermitian, so only the
//    n/2+1 samples with r >= 0 (plus r = -1/2) are gathered, samples with
//    x0 < 0 are taken at -p and conjugated, and the r-IFFT + c1dfftshift +
//    .real/4 collapse into one C2R of length n whose input index k holds
//    sample j = (k + n/2) mod n with sign (-1)^j / (4 n^2).
//  * RT is the exact transpose of that R.  The scatter is a pull over a
//    static CSR table (destination cell -> (sample, weight, conj)) built once
//    by a radix sort of (cell, sample, tap) keys: deterministic, no atomics
//    (tomo_scatter.cu).  The 4096-point column transforms are in tomo_col.cu.
#include "mm_common.cuh"
#include "fft_smem.cuh"
#include "tomo_kernels.cuh"
#include "tomo_int.cuh"

#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <type_traits>
#include <vector>

using mm::dev_alloc;

namespace {

// --------------------------------------------------------------------------
// R stage 1: padded phi*obj rows (processing/tomo.py:129-132, x padding only;
// the y padding lives in the zero rows of Y).
__global__ void k_pad_phi(const float* __restrict__ obj, float* __restrict__ P,
                          const float* __restrict__ phi1, float phis, int n, int nzc) {
    const long row = blockIdx.x;          // z * n + y
    const int y = (int)(row % n);
    const int z = (int)(row / n);
    const int twon = 2 * n, h = n / 2;
    float* out = P + row * twon;
    const bool live = z < nzc;
    const float* src = obj + row * n;
    const float py = phis * __ldg(phi1 + y);
    for (int x2 = threadIdx.x; x2 < twon; x2 += blockDim.x) {
        const int x = x2 - h;
        float v = 0.f;
        if (live && x >= 0 && x < n) v = py * __ldg(phi1 + x) * __ldg(src + x);
        out[x2] = v;
    }
}

// R stage 3: X[z][y][u] -> Y[n/2 + y][u][z]
__global__ void k_transpose_in(const float2* __restrict__ X, float2* __restrict__ Y, int n, int zs) {
    __shared__ float2 tile[32][33];
    const int u0 = blockIdx.x * 32, z0 = blockIdx.y * 32, y = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int j = ty; j < 32; j += 8) {
        const int z = z0 + j, u = u0 + tx;
        if (z < zs && u <= n) tile[j][tx] = __ldg(X + ((long)z * n + y) * (n + 1) + u);
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int u = u0 + j, z = z0 + tx;
        if (u <= n && z < zs) Y[((long)(y + n / 2) * (n + 1) + u) * zs + z] = tile[tx][j];
    }
}

// RT stage: B[n/2 + y][u][z] -> X[z][y][u], halving the interior columns
// (transpose of the R2C along x: the C2R counts them twice).
__global__ void k_transpose_out(const float2* __restrict__ B, float2* __restrict__ X, int n, int zs) {
    __shared__ float2 tile[32][33];
    const int u0 = blockIdx.x * 32, z0 = blockIdx.y * 32, y = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int j = ty; j < 32; j += 8) {
        const int u = u0 + j, z = z0 + tx;
        if (u <= n && z < zs) tile[j][tx] = __ldg(B + ((long)(y + n / 2) * (n + 1) + u) * zs + z);
    }
    __syncthreads();
    for (int j = ty; j < 32; j += 8) {
        const int z = z0 + j, u = u0 + tx;
        if (z < zs && u <= n) {
            float2 v = tile[tx][j];
            // the C2R reads only the real part of its DC and Nyquist bins; cuFFT
            // leaves the imaginary part's effect undefined, so clear it here
            if (u > 0 && u < n) { v.x *= 0.5f; v.y *= 0.5f; } else { v.y = 0.f; }
            X[((long)z * n + y) * (n + 1) + u] = v;
        }
    }
}

// R stage 4 / RT y-IFFT: length-2n transforms along v of the slice-
// interleaved spectrum, 4 adjacent (u, z) columns per block so every row
// access is one 32-byte sector.  Forward: rows outside [n/2, 3n/2) are the
// zero padding and are not read.  Inverse: only rows [n/2, 3n/2) are stored
// (the x-C2R needs nothing else).  src/dst row stride = (n+1)*zs.
// Forward: the gather reads only cells within radius n + m + 2 of the
// spectrum origin (polar samples have |p| <= n cells, windows reach m + 1
// further, reflected taps included), so rows outside radius n + 16 of each
// column are not stored (about a fifth of the half plane).  Inverse: the
// scatter leaves those cells unwritten (they receive nothing), so they are
// read as zeros.
// ZSC: zs fixed at compile time (then the row stride (n+1)*zs is too), 0 for runtime.
// Schedule width of the x-side forward and column transforms: 6144-point
// lines (n = 3072) take the wide 3 * 2^k schedule (48 values per thread), so
// that a column block holds four columns (32-byte row segments) at 512
// threads; measured 4.34 -> 3.85 ms forward column, 4.39 -> 4.02 ms inverse,
// 2.06 -> 1.87 ms x side at n = 3072.  (The x-side inverse keeps the default
// schedule: at 48 values per thread it needs 244 registers and ran slower.)
template <int L>
constexpr int xcol_vw() {
    return (!stockham::Sched<L>::P2 && L >= 6144) ? 48 : 0;
}
template <int L>
using ColSched = stockham::Sched<L, false, xcol_vw<L>()>;

// Columns per block: four, two where four would exceed 512 threads.
template <int L>
constexpr int col_cw() {
    return (!ColSched<L>::P2 && 4 * ColSched<L>::G > 512) ? 2 : 4;
}

template <int L, bool INV, int ZSC>
__global__ void __launch_bounds__(col_cw<L>() * ColSched<L>::G) k_col_fft(const float2* __restrict__ src,
                                                                              float2* __restrict__ dst,
                                                                              const float2* __restrict__ tw,
                                                                              long ncols_rt, int zs_rt) {
    namespace sk = stockham;
    constexpr int CW = col_cw<L>();
    const int zs = ZSC > 0 ? ZSC : zs_rt;
    const long ncols = ZSC > 0 ? (long)(L / 2 + 1) * ZSC : ncols_rt;
    extern __shared__ float2 sm[];
    const int c = threadIdx.x, g = threadIdx.y;
    const long col = (long)blockIdx.x * CW + c;
    const bool live = col < ncols;
    const int n = L / 2;
    const sk::ColAddr<CW> ad{c};
    const int u = (int)col / zs;
    const int r2max = (n + 16) * (n + 16) - u * u;
    auto ld = [&](int pos) -> float2 {
        if (!INV && (pos < n / 2 || pos >= 3 * n / 2)) return make_float2(0.f, 0.f);
        if (INV) {
            const int vw = pos < n ? pos : pos - L;
            if (vw * vw > r2max) return make_float2(0.f, 0.f);
        }
        return live ? __ldg(src + (long)pos * ncols + col) : make_float2(0.f, 0.f);
    };
    auto st = [&](int pos, float2 v) {
        if (INV && (pos < n / 2 || pos >= 3 * n / 2)) return;
        if (!INV) {
            const int vw = pos < n ? pos : pos - L;
            if (vw * vw > r2max) return;
        }
        if (live) dst[(long)pos * ncols + col] = v;
    };
    sk::fft<L, INV, xcol_vw<L>()>(sm, ad, ld, st, g, tw);
}

// ---------------------------------------------------------------------------
// Fused x-side and r-side transforms (Stockham lines in shared memory).

// Complex lines per x-side block: each line packs two rows (slices), so a
// block covers 2 * x_lines() slices = one 8 * 2 * x_lines()-byte segment per
// (v, u) of the slice-interleaved spectrum.
template <int L>
constexpr int x_lines() {
    return 2;
}
// Blocks per SM the inverse x side is compiled for (64 registers at two).
template <int L>
constexpr int x_min_blocks() {
    return (stockham::Sched<L>::P2 && x_lines<L>() * stockham::Sched<L>::G <= 512) ? 2 : 1;
}

// R x-side: rows (z, y) of phi*obj, zero padded to L = 2n, real FFT with two
// rows packed per complex line, written slice-interleaved into the centre
// rows of Y[v][u][z] (2 NL slices = one 16 NL-byte segment per u).
// Block (G, NL): line l holds rows z0 + 2l (real part) and z0 + 2l + 1 (imag).
template <int L, typename TIN>
__global__ void __launch_bounds__(x_lines<L>() * ColSched<L>::G) k_xfwd(const TIN* __restrict__ obj,
                                                                                float2* __restrict__ Y,
                                                                                const float* __restrict__ phi1,
                                                                                float phis,
                                                                                const float2* __restrict__ tw,
                                                                                int nzc, int zs) {
    constexpr int n = L / 2, LP = L + L / 16, G = ColSched<L>::G, NL = x_lines<L>(), ZB = 2 * NL;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x, l = threadIdx.y;
    const int y = blockIdx.y, z0 = blockIdx.x * ZB;  // z-groups fastest: a (v, u) segment fills at once
    const int za = z0 + 2 * l, zb = za + 1;
    const stockham::RowAddr ad{l * LP};
    const float py = phis * __ldg(phi1 + y);
    const TIN* ra = obj + ((long)za * n + y) * n;
    const TIN* rb = obj + ((long)zb * n + y) * n;
    auto ld = [&](int pos) -> float2 {
        const int x = pos - n / 2;
        if (x < 0 || x >= n) return make_float2(0.f, 0.f);
        const float w = py * __ldg(phi1 + x);
        return make_float2(za < nzc ? w * ld_elem(ra + x) : 0.f, zb < nzc ? w * ld_elem(rb + x) : 0.f);
    };
    auto st = [&](int pos, float2 v) { sm[ad(pos)] = v; };
    stockham::fft<L, false, xcol_vw<L>()>(sm, ad, ld, st, g, tw);
    __syncthreads();
    const int tid = l * G + g;
    const int nq = min(ZB, zs - z0);
    // NL lanes per u, lane h storing line h's two slices (16 bytes): a warp
    // store covers 32/NL whole segments instead of 32 half segments, half the
    // L1 wavefronts of one lane per u
    for (int idx = tid; idx < NL * (n + 1); idx += NL * G) {
        const int k = idx / NL, h = idx % NL;
        const int km = k == 0 ? 0 : L - k;
        const float2 zk = sm[h * LP + k + (k >> 4)];
        const float2 zm = sm[h * LP + km + (km >> 4)];
        // A = (Zk + conj Zm)/2 (real row), B = (Zk - conj Zm)/(2i) (imag row)
        const float2 A = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 Bv = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
        float2* dst = Y + ((long)(y + n / 2) * (n + 1) + k) * zs + z0 + 2 * h;
        if (2 * h + 1 < nq) reinterpret_cast<float4*>(dst)[0] = make_float4(A.x, A.y, Bv.x, Bv.y);
        else if (2 * h < nq) dst[0] = A;
    }
}

// RT x-side: centre rows of B[v][u][z] for one y and 2 NL slices -> halve
// the interior columns (transpose of the x real FFT), real parts only at
// u = 0 and u = n, two rows packed per complex inverse line, crop to
// [n/2, 3n/2), times phi.  OUT 0: float obj; 1/2: real/imag part of complex.
template <int L, int OUT, typename TOUT = float>
__global__ void __launch_bounds__(x_lines<L>() * stockham::Sched<L>::G, x_min_blocks<L>())
    k_xinv(const float2* __restrict__ B, void* __restrict__ obj, const float* __restrict__ phi1, float phis,
           const float2* __restrict__ tw, int nzc, int zs) {
    constexpr int n = L / 2, LP = L + L / 16, G = stockham::Sched<L>::G, NL = x_lines<L>(), ZB = 2 * NL;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x, l = threadIdx.y;
    const int y = blockIdx.y, z0 = blockIdx.x * ZB;  // z-groups fastest: a (v, u) segment fills at once
    const int tid = l * G + g;
    const int nq = min(ZB, zs - z0);
    // one thread per u: load the slices (one contiguous segment), line h
    // gets Z = A + iB from rows 2h (A) and 2h + 1 (B).  (Two lanes per u as
    // in k_xfwd's stores measured 1.31 -> 1.32 ms here, and slower at 6144.)
    for (int k = tid; k <= n; k += NL * G) {
        const float2* src = B + ((long)(y + n / 2) * (n + 1) + k) * zs + z0;
        float2 v[ZB];
        if (nq == ZB) {
#pragma unroll
            for (int h = 0; h < NL; ++h) {
                const float4 a = __ldg(reinterpret_cast<const float4*>(src) + h);
                v[2 * h] = make_float2(a.x, a.y);
                v[2 * h + 1] = make_float2(a.z, a.w);
            }
        } else {
            for (int q = 0; q < ZB; ++q) v[q] = q < nq ? __ldg(src + q) : make_float2(0.f, 0.f);
        }
        const bool interior = k > 0 && k < n;
#pragma unroll
        for (int q = 0; q < ZB; ++q) {
            if (interior) { v[q].x *= 0.5f; v[q].y *= 0.5f; } else { v[q].y = 0.f; }
        }
#pragma unroll
        for (int h = 0; h < NL; ++h) {
            const float2 A = v[2 * h], Bv = v[2 * h + 1];
            sm[h * LP + k + (k >> 4)] = make_float2(A.x - Bv.y, A.y + Bv.x);              // A + iB
            if (interior) {
                const int km = L - k;
                sm[h * LP + km + (km >> 4)] = make_float2(A.x + Bv.y, Bv.x - A.y);        // conj A + i conj B
            }
        }
    }
    __syncthreads();
    const stockham::RowAddr ad{l * LP};
    const int za = z0 + 2 * l, zb = za + 1;
    const float py = phis * __ldg(phi1 + y);
    auto ld = [&](int pos) -> float2 { return sm[ad(pos)]; };
    auto st = [&](int pos, float2 v) {
        const int x = pos - n / 2;
        if (x < 0 || x >= n) return;
        const float w = py * __ldg(phi1 + x);
        if (OUT == 0) {
            TOUT* o = static_cast<TOUT*>(obj);
            if (za < nzc) st_elem(o + ((long)za * n + y) * n + x, w * v.x);
            if (zb < nzc) st_elem(o + ((long)zb * n + y) * n + x, w * v.y);
        } else {
            float* o = static_cast<float*>(obj);
            if (za < nzc) o[(((long)za * n + y) * n + x) * 2 + (OUT - 1)] = w * v.x;
            if (zb < nzc) o[(((long)zb * n + y) * n + x) * 2 + (OUT - 1)] = w * v.y;
        }
    };
    stockham::fft<L, true>(sm, ad, ld, st, g, tw);
}

// R r-side: C2R of length 2M along k for columns c of H[k][c] (k = 0..M),
// as a complex inverse line of M points: Z[k] = (X[k] + conj X[M-k]) +
// i e^{+2 pi i k/2M} (X[k] - conj X[M-k]); x[2m] = Re z[m], x[2m+1] = Im z[m].
// Block (G, 8): eight columns (64 bytes per k) per block.
template <int M, typename TOUT>
__global__ void __launch_bounds__(8 * stockham::Sched<M>::G, stockham::Sched<M>::P2 ? 2 : 1) k_rc2r(const float2* __restrict__ H,
                                                                     TOUT* __restrict__ out,
                                                                     const float2* __restrict__ tw,
                                                                     const float2* __restrict__ ex, long C) {
    constexpr int CB = 8, LP = M + M / 16, G = stockham::Sched<M>::G;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x, l = threadIdx.y;
    const long c0 = (long)blockIdx.x * CB;
    const int tid = l * G + g;
    float2* stg = sm;  // [CB][M + 1]; aliased by the line buffers after pass 0 reads
    {
        // all loads of this thread issued before any store (latency bound)
        constexpr int PER = ((M + 1) * CB + CB * G - 1) / (CB * G);
        float2 v[PER];
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int idx = tid + r * CB * G;
            const int c = idx & (CB - 1), k = idx >> 3;
            v[r] = (idx < (M + 1) * CB && c0 + c < C) ? __ldg(H + (long)k * C + c0 + c) : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int idx = tid + r * CB * G;
            if (idx < (M + 1) * CB) stg[(idx & (CB - 1)) * (M + 1) + (idx >> 3)] = v[r];
        }
    }
    __syncthreads();
    const stockham::RowAddr ad{l * LP};
    const float2* X = stg + l * (M + 1);
    auto ld = [&](int pos) -> float2 {
        const float2 a = X[pos], b = X[M - pos];
        const float2 e = make_float2(a.x + b.x, a.y - b.y);            // X[k] + conj X[M-k]
        const float2 d = make_float2(a.x - b.x, a.y + b.y);            // X[k] - conj X[M-k]
        const float2 w = __ldg(ex + pos);                               // e^{+2 pi i k / 2M}
        const float2 od = make_float2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
        return make_float2(e.x - od.y, e.y + od.x);                     // e + i od
    };
    TOUT* orow = out + (c0 + l) * (2 * M);
    const bool live = c0 + l < C;
    auto st = [&](int pos, float2 v) {
        if (live) st_pair(orow + 2 * pos, v);
    };
    stockham::fft<M, true>(sm, ad, ld, st, g, tw);
}

// Columns (rows y[c]) per block of the RT r side.
template <int M>
constexpr int rr_cols() {
    return 8;
}

// RT r-side: R2C of length 2M of real rows y[c][0..2M) as a complex forward
// line z[m] = y[2m] + i y[2m+1]; X[k] = (Z[k] + conj Z[M-k])/2 +
// e^{-2 pi i k/2M} (Z[k] - conj Z[M-k])/(2i) for k = 0..M, written to
// H[k][c] (CB columns = 8 CB bytes per k).
template <int M, typename TIN>
__global__ void __launch_bounds__(rr_cols<M>() * stockham::Sched<M>::G) k_rr2c(const TIN* __restrict__ yv,
                                                                                float2* __restrict__ H,
                                                                                const float2* __restrict__ tw,
                                                                                const float2* __restrict__ ex,
                                                                                long C) {
    // odd line stride: the epilogue's CB lanes at one k read CB different
    // lines, which then fall in different banks
    constexpr int CB = rr_cols<M>(), LP = M + M / 16 + 1, G = stockham::Sched<M>::G;
    extern __shared__ float2 sm[];
    const int g = threadIdx.x, l = threadIdx.y;
    const long c0 = (long)blockIdx.x * CB;
    const bool live = c0 + l < C;
    const TIN* row = yv + (c0 + l) * (2 * M);
    const stockham::RowAddr ad{l * LP};
    auto ld = [&](int pos) -> float2 { return live ? ld_pair(row + 2 * pos) : make_float2(0.f, 0.f); };
    auto st = [&](int pos, float2 v) { sm[ad(pos)] = v; };
    stockham::fft<M, false>(sm, ad, ld, st, g, tw);
    __syncthreads();
    const int tid = l * G + g;
    for (int idx = tid; idx < (M + 1) * CB; idx += CB * G) {
        const int c = idx % CB, k = idx / CB;
        if (c0 + c >= C) continue;
        const int kk = k == M ? 0 : k, km = k == 0 ? 0 : M - k;
        const float2 a = sm[c * LP + kk + (kk >> 4)], b = sm[c * LP + km + (km >> 4)];
        const float2 e = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));     // (Zk + conj Zm)/2
        const float2 d = make_float2(0.5f * (a.y + b.y), 0.5f * (b.x - a.x));     // (Zk - conj Zm)/(2i)
        const float2 w = __ldg(ex + k);                                           // e^{+2 pi i k / 2M}
        const float2 od = make_float2(d.x * w.x + d.y * w.y, d.y * w.x - d.x * w.y);  // d * conj(w)
        H[(long)k * C + c0 + c] = make_float2(e.x + od.x, e.y + od.y);
    }
}

// The 2m+1 taps of window row v (columns bx .. bx+2m), all loads issued
// before any is used; taps outside the stored half plane are reflected and
// conjugated (tap_cell).
// ZSC: the slice count zs when fixed at compile time (tap offsets become
// immediates), 0 for a runtime zs.
template <int ZV, int M, int ZSC>
__device__ __forceinline__ void load_row(const float2* __restrict__ F, int bx, int v, bool fast, int n, int zs_rt,
                                         int zoff, float (&val)[2 * M + 1][2 * ZV]) {
    constexpr int L = 2 * M + 1;
    const int zs = ZSC > 0 ? ZSC : zs_rt;
    const long rowstride = (long)(n + 1) * zs;
    const int twon = 2 * n;
    if (fast) {
        const int row = v < 0 ? v + twon : (v >= twon ? v - twon : v);
        const float2* p = F + row * rowstride + (long)bx * zs + zoff;
#pragma unroll
        for (int i0 = 0; i0 < L; ++i0) ZVec<ZV>::load(p + (long)i0 * zs, val[i0]);
    } else {
#pragma unroll
        for (int i0 = 0; i0 < L; ++i0) {
            int row, col;
            bool cj;
            tap_cell(bx + i0, v, n, row, col, cj);
            ZVec<ZV>::load(F + row * rowstride + (long)col * zs + zoff, val[i0]);
            if (cj) {
#pragma unroll
                for (int q = 1; q < 2 * ZV; q += 2) val[i0][q] = -val[i0][q];
            }
        }
    }
}

// Window sum of one sample: (2m+1)^2 taps, row partial sums along x first.
template <int ZV, int M, int ZSC>
__device__ __forceinline__ void window_sum(const float2* __restrict__ F, const SampleGeo& g, const float* wx,
                                           const float* wy, float* acc, int n, int zs, int zoff) {
    constexpr int L = 2 * M + 1;
    const bool fast = (g.bx >= 0) && (g.bx + 2 * M <= n);
#pragma unroll
    for (int i1 = 0; i1 < L; ++i1) {
        float val[L][2 * ZV];
        load_row<ZV, M, ZSC>(F, g.bx, g.by + i1, fast, n, zs, zoff, val);
        float ar[2 * ZV];
#pragma unroll
        for (int q = 0; q < 2 * ZV; ++q) ar[q] = 0.f;
#pragma unroll
        for (int i0 = 0; i0 < L; ++i0) {
#pragma unroll
            for (int q = 0; q < 2 * ZV; ++q) ar[q] = fmaf(wx[i0], val[i0][q], ar[q]);
        }
#pragma unroll
        for (int q = 0; q < 2 * ZV; ++q) acc[q] = fmaf(wy[i1], ar[q], acc[q]);
    }
}

// Sign of the C2R input slot and store of one gathered sample.
template <int ZV>
__device__ __forceinline__ void store_sample(float2* __restrict__ H, const SampleGeo& g, float* acc, int k, int t,
                                             int n, int T, int zs, int zoff, float scale) {
    const float sc = (g.j & 1) ? -scale : scale;
    const float si = (k == 0 || k == n / 2) ? 0.f : (g.mir ? -sc : sc);
#pragma unroll
    for (int q = 0; q < 2 * ZV; q += 2) {
        acc[q] *= sc;
        acc[q + 1] *= si;
    }
    ZVec<ZV>::store(H + ((long)k * T + t) * zs + zoff, acc);
}

// R stage 5: Gaussian gather of the n/2+1 non-redundant samples per angle.
// One group of LPS lanes per sample; each lane owns ZV slices.
// Blocks per SM: 4 (64 registers) when the weights are spread over the lanes
// and the window is at most 9 x 9; else 3 for single samples (a few spills
// at m >= 4 when several samples share a warp, still faster than 2 blocks)
// and 2 for pairs.
template <int LPS, int M, bool PAIR>
constexpr int gather_min_blocks() {
    return (LPS == 32 && M <= 4) ? 4 : (PAIR ? 2 : 3);
}

template <int ZV, int LPS, int M, int ZSC>
__global__ void __launch_bounds__(kThreads, gather_min_blocks<LPS, M, false>()) k_gather(const float2* __restrict__ F, float2* __restrict__ H,
                                                     const float* __restrict__ cosT, const float* __restrict__ sinT,
                                                     int n, int T, int zs, float c0, float c1, float scale,
                                                     int clamp) {
    constexpr int L = 2 * M + 1;
    constexpr int SPW = 32 / LPS;
    const int K = n / 2 + 1;
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPS, zl = lane % LPS;
    const int zgroups = zs / (LPS * ZV);
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long zg = warp % zgroups;
    const long s = (warp / zgroups) * SPW + sub;
    if (s >= (long)T * K) return;
    // angle-major: consecutive warps take the same radius on consecutive
    // angles, whose windows overlap most (and whose H rows are adjacent)
    const int t = (int)(s % T), k = (int)(s / T);
    const SampleGeo g = sample_geo(t, k, n, M, cosT, sinT, clamp != 0);
    const float inv_twon = 1.0f / (float)(2 * n);
    float wx[L], wy[L];
    if constexpr (LPS == 32) {  // one sample per warp: weights spread over the lanes
        const WarpWeights<L, 1> ww(lane, g, g, inv_twon, c0, c1);
#pragma unroll
        for (int i = 0; i < L; ++i) {
            wx[i] = ww.get(i);
            wy[i] = ww.get(L + i);
        }
    } else {
#pragma unroll
        for (int i = 0; i < L; ++i) {
            wx[i] = tap_weight(g.bx + i, g.x0, inv_twon, c1);
            wy[i] = c0 * tap_weight(g.by + i, g.y0, inv_twon, c1);
        }
    }
    const int zoff = (int)zg * (LPS * ZV) + zl * ZV;
    float acc[2 * ZV];
#pragma unroll
    for (int q = 0; q < 2 * ZV; ++q) acc[q] = 0.f;
    window_sum<ZV, M, ZSC>(F, g, wx, wy, acc, n, zs, zoff);
    // k = 0 and k = n/2 are the DC and Nyquist bins of the C2R along r: only
    // their real part enters the result (the .real of tomo.py:150)
    store_sample<ZV>(H, g, acc, k, t, n, T, zs, zoff, scale);
}

// R stage 5 for angle sets symmetric under theta -> theta + pi (T even,
// theta[t + T/2] = theta[t] + pi up to float32 rounding): the sample at radius
// k of angle t + T/2 lies at the negated frequency of angle t's, which the
// Hermitian fold maps back onto the same point, so the two usually share
// their (2m+1)^2 window.  One lane group takes both samples; when the windows
// coincide every tap is loaded once and weighted with each sample's own
// weights, otherwise the two windows are summed one after the other.  Each
// sample's arithmetic is exactly k_gather's (window_sum, store_sample).
template <int ZV, int LPS, int M, int ZSC>
__global__ void __launch_bounds__(kThreads, gather_min_blocks<LPS, M, true>()) k_gather_pair(const float2* __restrict__ F, float2* __restrict__ H,
                                                          const float* __restrict__ cosT,
                                                          const float* __restrict__ sinT, int n, int T, int zs,
                                                          float c0, float c1, float scale, int clamp) {
    constexpr int L = 2 * M + 1;
    constexpr int SPW = 32 / LPS;
    const int K = n / 2 + 1, T2 = T / 2;
    const int lane = threadIdx.x & 31;
    const int sub = lane / LPS, zl = lane % LPS;
    const int zgroups = zs / (LPS * ZV);
    const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long zg = warp % zgroups;
    const long s = (warp / zgroups) * SPW + sub;
    if (s >= (long)T2 * K) return;
    const int t = (int)(s % T2), k = (int)(s / T2);
    const SampleGeo ga = sample_geo(t, k, n, M, cosT, sinT, clamp != 0);
    const SampleGeo gb = sample_geo(t + T2, k, n, M, cosT, sinT, clamp != 0);
    const float inv_twon = 1.0f / (float)(2 * n);
    float wxa[L], wya[L], wxb[L], wyb[L];
    if constexpr (LPS == 32) {  // one pair per warp: weights spread over the lanes
        const WarpWeights<L, 2> ww(lane, ga, gb, inv_twon, c0, c1);
#pragma unroll
        for (int i = 0; i < L; ++i) {
            wxa[i] = ww.get(i);
            wya[i] = ww.get(L + i);
            wxb[i] = ww.get(2 * L + i);
            wyb[i] = ww.get(3 * L + i);
        }
    } else {
#pragma unroll
        for (int i = 0; i < L; ++i) {
            wxa[i] = tap_weight(ga.bx + i, ga.x0, inv_twon, c1);
            wya[i] = c0 * tap_weight(ga.by + i, ga.y0, inv_twon, c1);
            wxb[i] = tap_weight(gb.bx + i, gb.x0, inv_twon, c1);
            wyb[i] = c0 * tap_weight(gb.by + i, gb.y0, inv_twon, c1);
        }
    }
    const int zoff = (int)zg * (LPS * ZV) + zl * ZV;
    float acca[2 * ZV], accb[2 * ZV];
#pragma unroll
    for (int q = 0; q < 2 * ZV; ++q) acca[q] = accb[q] = 0.f;
    if (ga.bx == gb.bx && ga.by == gb.by) {
        const bool fast = (ga.bx >= 0) && (ga.bx + 2 * M <= n);
#pragma unroll
        for (int i1 = 0; i1 < L; ++i1) {
            float val[L][2 * ZV];
            load_row<ZV, M, ZSC>(F, ga.bx, ga.by + i1, fast, n, zs, zoff, val);
            float ara[2 * ZV], arb[2 * ZV];
#pragma unroll
            for (int q = 0; q < 2 * ZV; ++q) ara[q] = arb[q] = 0.f;
#pragma unroll
            for (int i0 = 0; i0 < L; ++i0) {
#pragma unroll
                for (int q = 0; q < 2 * ZV; ++q) {
                    ara[q] = fmaf(wxa[i0], val[i0][q], ara[q]);
                    arb[q] = fmaf(wxb[i0], val[i0][q], arb[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < 2 * ZV; ++q) {
                acca[q] = fmaf(wya[i1], ara[q], acca[q]);
                accb[q] = fmaf(wyb[i1], arb[q], accb[q]);
            }
        }
    } else {
        window_sum<ZV, M, ZSC>(F, ga, wxa, wya, acca, n, zs, zoff);
        window_sum<ZV, M, ZSC>(F, gb, wxb, wyb, accb, n, zs, zoff);
    }
    store_sample<ZV>(H, ga, acca, k, t, n, T, zs, zoff, scale);
    store_sample<ZV>(H, gb, accb, k, t + T2, n, T, zs, zoff, scale);
}

// RT final stage: obj = phi * crop(Q); OUT = 0 real, 1/2 real/imag part of c64.
template <int OUT>
__global__ void k_crop_phi(const float* __restrict__ Q, void* __restrict__ obj, const float* __restrict__ phi1,
                           float phis, int n) {
    const long row = blockIdx.x;  // z * n + y
    const int y = (int)(row % n);
    const float py = phis * __ldg(phi1 + y);
    const float* src = Q + row * 2 * n + n / 2;
    for (int x = threadIdx.x; x < n; x += blockDim.x) {
        const float v = py * __ldg(phi1 + x) * __ldg(src + x);
        if (OUT == 0)
            static_cast<float*>(obj)[row * n + x] = v;
        else
            static_cast<float*>(obj)[(row * n + x) * 2 + (OUT - 1)] = v;
    }
}

// (T, zs, n) -> (T, nzc, n) and back, zero-filling the extra slices.
__global__ void k_copy_z(const float* __restrict__ src, float* __restrict__ dst, int n, int zsrc, int zdst,
                         int zvalid) {
    const long row = blockIdx.x;  // t * zdst + z
    const int z = (int)(row % zdst);
    const long t = row / zdst;
    float* d = dst + row * n;
    const float* s = src + (t * zsrc + z) * n;
    for (int x = threadIdx.x; x < n; x += blockDim.x) d[x] = (z < zvalid) ? __ldg(s + x) : 0.f;
}
template <typename TI, typename TO>
__global__ void k_copy_z_t(const TI* __restrict__ src, TO* __restrict__ dst, int n, int zsrc, int zdst,
                           int zvalid) {
    const long row = blockIdx.x;  // t * zdst + z
    const int z = (int)(row % zdst);
    const long t = row / zdst;
    TO* d = dst + row * n;
    const TI* s = src + (t * zsrc + z) * n;
    for (int x = threadIdx.x; x < n; x += blockDim.x) st_elem(d + x, (z < zvalid) ? ld_elem(s + x) : 0.f);
}

__global__ void k_copy_z_c(const float2* __restrict__ src, float2* __restrict__ dst, int n, int zsrc, int zdst,
                           int zvalid) {
    const long row = blockIdx.x;
    const int z = (int)(row % zdst);
    const long t = row / zdst;
    float2* d = dst + row * n;
    const float2* s = src + (t * zsrc + z) * n;
    for (int x = threadIdx.x; x < n; x += blockDim.x) d[x] = (z < zvalid) ? __ldg(s + x) : make_float2(0.f, 0.f);
}

// Complex RT: Hermitian (PART=0) or anti-Hermitian times -i (PART=1) part of
// the line spectra, in the scatter's input layout Q[k][t][z].
template <int PART>
__global__ void k_combine(const float2* __restrict__ Yc, float2* __restrict__ Q, int n, int T, int zs) {
    const long row = blockIdx.x;  // t * zs + z
    const int z = (int)(row % zs);
    const long t = row / zs;
    const float2* y = Yc + row * n;
    const int K = n / 2 + 1;
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const float2 a = __ldg(y + k);
        float2 q;
        if (k == 0 || k == n / 2) {
            q = a;
        } else {
            const float2 b = __ldg(y + (n - k));
            q = PART == 0 ? make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y))
                          : make_float2(0.5f * (a.x - b.x), 0.5f * (a.y + b.y));
        }
        if (PART == 1) q = make_float2(q.y, -q.x);  // times -i
        Q[((long)k * T + t) * zs + z] = q;
    }
}

// --------------------------------------------------------------------------
int plan1d(cufftHandle* plan, long long len, long long istride, long long idist, long long ostride,
           long long odist, cufftType type, long long batch, size_t* work) {
    MM_CUFFT(cufftCreate(plan));
    MM_CUFFT(cufftSetAutoAllocation(*plan, 0));
    long long nn[1] = {len};
    const bool r2c = type == CUFFT_R2C, c2r = type == CUFFT_C2R;
    long long inemb[1] = {c2r ? len / 2 + 1 : len};
    long long onemb[1] = {r2c ? len / 2 + 1 : len};
    size_t ws = 0;
    MM_CUFFT(cufftMakePlanMany64(*plan, 1, nn, inemb, istride, idist, onemb, ostride, odist, type, batch, &ws));
    *work = std::max(*work, ws);
    return MM_OK;
}

// One work area shared by every cuFFT plan of the handle (they run in
// sequence on one stream); grown when a new plan needs more, and attached to
// every plan each time a plan is added.
int ensure_work(mm_tomo* h, size_t need) {
    if (need == 0 && !h->fft_work) return MM_OK;  // no cuFFT plan needs scratch
    if (need > h->fft_work_bytes || !h->fft_work) {
        if (h->fft_work) {
            cudaFree(h->fft_work);
            h->ws_bytes -= h->fft_work_bytes;
            h->fft_work = nullptr;
            h->fft_work_bytes = 0;
        }
        MM_TRY(dev_alloc(&h->fft_work, need, "cuFFT work area"));
        h->fft_work_bytes = need;
        h->ws_bytes += need;
    }
    cufftHandle all[6] = {h->plan_xr2c, h->plan_xc2r, h->plan_y, h->plan_rc2r, h->plan_rr2c, h->plan_rc2c};
    for (cufftHandle p : all)
        if (p) MM_CUFFT(cufftSetWorkArea(p, h->fft_work));
    return MM_OK;
}


template <int L, bool INV>
int launch_col_fft_l(mm_tomo* h, const float2* src, float2* dst, cudaStream_t st) {
    namespace sk = stockham;
    constexpr int CW = col_cw<L>(), G = ColSched<L>::G;
    const long ncols = (long)(h->n + 1) * h->zs;
    const size_t smem = (size_t)sk::ColAddr<CW>::rows(L) * CW * sizeof(float2);
    // 3 * 2^k lengths: runtime slice count only (one instantiation each)
    auto kern = (sk::Sched<L>::P2 && h->zs == 64) ? k_col_fft<L, INV, sk::Sched<L>::P2 ? 64 : 0> : k_col_fft<L, INV, 0>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 block(CW, G), grid((unsigned)((ncols + CW - 1) / CW));
    kern<<<grid, block, smem, st>>>(src, dst, xcol_vw<L>() ? h->d_tww : h->d_twy, ncols, h->zs);
    MM_LAUNCHED();
    return MM_OK;
}

// Column transform along v (length 2n) of the slice-interleaved spectrum:
// the 64 x 64 kernel with full-line accesses (tomo_col.cu) where it applies,
// else one shared-memory block per four columns.
template <bool INV>
int launch_col_fft(mm_tomo* h, const float2* src, float2* dst, cudaStream_t st) {
    const int rc = mmtomo::col_fft_pipe(h->n, h->zs, INV, src, dst, h->col_scratch, h->col_tw, h->sms, st);
    if (rc != mmtomo::kNotCovered) return rc;
    switch (2 * h->n) {
        case 16: return launch_col_fft_l<16, INV>(h, src, dst, st);
        case 32: return launch_col_fft_l<32, INV>(h, src, dst, st);
        case 64: return launch_col_fft_l<64, INV>(h, src, dst, st);
        case 128: return launch_col_fft_l<128, INV>(h, src, dst, st);
        case 256: return launch_col_fft_l<256, INV>(h, src, dst, st);
        case 512: return launch_col_fft_l<512, INV>(h, src, dst, st);
        case 1024: return launch_col_fft_l<1024, INV>(h, src, dst, st);
        case 2048: return launch_col_fft_l<2048, INV>(h, src, dst, st);
        case 4096: return launch_col_fft_l<4096, INV>(h, src, dst, st);
        case 96: return launch_col_fft_l<96, INV>(h, src, dst, st);
        case 192: return launch_col_fft_l<192, INV>(h, src, dst, st);
        case 384: return launch_col_fft_l<384, INV>(h, src, dst, st);
        case 768: return launch_col_fft_l<768, INV>(h, src, dst, st);
        case 1536: return launch_col_fft_l<1536, INV>(h, src, dst, st);
        case 3072: return launch_col_fft_l<3072, INV>(h, src, dst, st);
        case 6144: return launch_col_fft_l<6144, INV>(h, src, dst, st);
    }
    return -100;  // no native kernel for this length: caller uses cuFFT
}

template <int L, typename TIN>
int launch_xfwd_l(mm_tomo* h, const void* obj, int nzc, cudaStream_t st) {
    constexpr int G = ColSched<L>::G, NL = x_lines<L>();
    const size_t smem = (size_t)NL * (L + L / 16) * sizeof(float2);
    auto kern = k_xfwd<L, TIN>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 block(G, NL), grid((h->zs + 2 * NL - 1) / (2 * NL), h->n);
    kern<<<grid, block, smem, st>>>((const TIN*)obj, h->Y, h->d_phi1, h->phi_scale,
                                    xcol_vw<L>() ? h->d_tww : h->d_twy, nzc, h->zs);
    MM_LAUNCHED();
    return MM_OK;
}

template <int L, int OUT, typename TOUT>
int launch_xinv_l(mm_tomo* h, void* obj, int nzc, cudaStream_t st) {
    constexpr int G = stockham::Sched<L>::G, NL = x_lines<L>();
    const size_t smem = (size_t)NL * (L + L / 16) * sizeof(float2);
    auto kern = k_xinv<L, OUT, TOUT>;
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 block(G, NL), grid((h->zs + 2 * NL - 1) / (2 * NL), h->n);
    kern<<<grid, block, smem, st>>>(h->Y, obj, h->d_phi1, h->phi_scale, h->d_twy, nzc, h->zs);
    MM_LAUNCHED();
    return MM_OK;
}

template <int M, typename TS>
int launch_r_l(mm_tomo* h, bool inv, const void* src, void* dst, cudaStream_t st) {
    constexpr int G = stockham::Sched<M>::G;
    const size_t smem = (size_t)8 * (M + M / 16 > M + 1 ? M + M / 16 : M + 1) * sizeof(float2);
    const long C = (long)h->ntheta * h->zs;
    dim3 block(G, 8), grid((unsigned)((C + 7) / 8));
    if (inv) {
        auto kern = k_rc2r<M, TS>;
        MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<grid, block, smem, st>>>((const float2*)src, (TS*)dst, h->d_twr, h->d_exr, C);
    } else {
        constexpr int CBr = rr_cols<M>();
        const size_t smem_r = (size_t)CBr * (M + M / 16 + 1) * sizeof(float2);
        auto kern = k_rr2c<M, TS>;
        MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_r));
        kern<<<dim3((unsigned)((C + CBr - 1) / CBr)), dim3(G, CBr), smem_r, st>>>((const TS*)src, (float2*)dst,
                                                                                 h->d_twr, h->d_exr, C);
    }
    MM_LAUNCHED();
    return MM_OK;
}

template <typename TIN>
int launch_xfwd_t(mm_tomo* h, const void* obj, int nzc, cudaStream_t st) {
    switch (2 * h->n) {
        case 64: return launch_xfwd_l<64, TIN>(h, obj, nzc, st);
        case 128: return launch_xfwd_l<128, TIN>(h, obj, nzc, st);
        case 256: return launch_xfwd_l<256, TIN>(h, obj, nzc, st);
        case 512: return launch_xfwd_l<512, TIN>(h, obj, nzc, st);
        case 1024: return launch_xfwd_l<1024, TIN>(h, obj, nzc, st);
        case 2048: return launch_xfwd_l<2048, TIN>(h, obj, nzc, st);
        case 4096: return launch_xfwd_l<4096, TIN>(h, obj, nzc, st);
    }
    if constexpr (std::is_same<TIN, float>::value) {  // 3 * 2^k lengths: float32 storage only
        switch (2 * h->n) {
            case 96: return launch_xfwd_l<96, TIN>(h, obj, nzc, st);
            case 192: return launch_xfwd_l<192, TIN>(h, obj, nzc, st);
            case 384: return launch_xfwd_l<384, TIN>(h, obj, nzc, st);
            case 768: return launch_xfwd_l<768, TIN>(h, obj, nzc, st);
            case 1536: return launch_xfwd_l<1536, TIN>(h, obj, nzc, st);
            case 3072: return launch_xfwd_l<3072, TIN>(h, obj, nzc, st);
            case 6144: return launch_xfwd_l<6144, TIN>(h, obj, nzc, st);
        }
    }
    MM_REQUIRE(false, "x transform: unsupported n=%d", h->n);
}

int launch_xfwd(mm_tomo* h, const void* obj, int dtype, int nzc, cudaStream_t st) {
    return dtype == MM_BF16 ? launch_xfwd_t<__nv_bfloat16>(h, obj, nzc, st) : launch_xfwd_t<float>(h, obj, nzc, st);
}

template <int OUT, typename TOUT>
int launch_xinv_t(mm_tomo* h, void* obj, int nzc, cudaStream_t st) {
    switch (2 * h->n) {
        case 64: return launch_xinv_l<64, OUT, TOUT>(h, obj, nzc, st);
        case 128: return launch_xinv_l<128, OUT, TOUT>(h, obj, nzc, st);
        case 256: return launch_xinv_l<256, OUT, TOUT>(h, obj, nzc, st);
        case 512: return launch_xinv_l<512, OUT, TOUT>(h, obj, nzc, st);
        case 1024: return launch_xinv_l<1024, OUT, TOUT>(h, obj, nzc, st);
        case 2048: return launch_xinv_l<2048, OUT, TOUT>(h, obj, nzc, st);
        case 4096: return launch_xinv_l<4096, OUT, TOUT>(h, obj, nzc, st);
    }
    if constexpr (std::is_same<TOUT, float>::value) {  // 3 * 2^k lengths: float32 storage only
        switch (2 * h->n) {
            case 96: return launch_xinv_l<96, OUT, TOUT>(h, obj, nzc, st);
            case 192: return launch_xinv_l<192, OUT, TOUT>(h, obj, nzc, st);
            case 384: return launch_xinv_l<384, OUT, TOUT>(h, obj, nzc, st);
            case 768: return launch_xinv_l<768, OUT, TOUT>(h, obj, nzc, st);
            case 1536: return launch_xinv_l<1536, OUT, TOUT>(h, obj, nzc, st);
            case 3072: return launch_xinv_l<3072, OUT, TOUT>(h, obj, nzc, st);
            case 6144: return launch_xinv_l<6144, OUT, TOUT>(h, obj, nzc, st);
        }
    }
    MM_REQUIRE(false, "x transform: unsupported n=%d", h->n);
}

template <int OUT>
int launch_xinv(mm_tomo* h, void* obj, int nzc, cudaStream_t st, int dtype = MM_F32) {
    if (OUT == 0 && dtype == MM_BF16) return launch_xinv_t<0, __nv_bfloat16>(h, obj, nzc, st);
    return launch_xinv_t<OUT, float>(h, obj, nzc, st);
}

template <typename TS>
int launch_r_t(mm_tomo* h, bool inv, const void* src, void* dst, cudaStream_t st) {
    switch (h->n / 2) {
        case 16: return launch_r_l<16, TS>(h, inv, src, dst, st);
        case 32: return launch_r_l<32, TS>(h, inv, src, dst, st);
        case 64: return launch_r_l<64, TS>(h, inv, src, dst, st);
        case 128: return launch_r_l<128, TS>(h, inv, src, dst, st);
        case 256: return launch_r_l<256, TS>(h, inv, src, dst, st);
        case 512: return launch_r_l<512, TS>(h, inv, src, dst, st);
        case 1024: return launch_r_l<1024, TS>(h, inv, src, dst, st);
        case 2048: return launch_r_l<2048, TS>(h, inv, src, dst, st);
    }
    if constexpr (std::is_same<TS, float>::value) {  // 3 * 2^k lengths: float32 storage only
        switch (h->n / 2) {
            case 24: return launch_r_l<24, TS>(h, inv, src, dst, st);
            case 48: return launch_r_l<48, TS>(h, inv, src, dst, st);
            case 96: return launch_r_l<96, TS>(h, inv, src, dst, st);
            case 192: return launch_r_l<192, TS>(h, inv, src, dst, st);
            case 384: return launch_r_l<384, TS>(h, inv, src, dst, st);
            case 768: return launch_r_l<768, TS>(h, inv, src, dst, st);
            case 1536: return launch_r_l<1536, TS>(h, inv, src, dst, st);
        }
    }
    MM_REQUIRE(false, "r transform: unsupported n=%d", h->n);
}

// r-side transform; `dtype` is the storage type of the real sinogram side.
int launch_r(mm_tomo* h, bool inv, const void* src, void* dst, cudaStream_t st, int dtype = MM_F32) {
    return dtype == MM_BF16 ? launch_r_t<__nv_bfloat16>(h, inv, src, dst, st) : launch_r_t<float>(h, inv, src, dst, st);
}


template <int ZV, int LPS, int ZSC>
int launch_gather_m(mm_tomo* h, cudaStream_t st) {
    const int K = h->K;
    const long samples = (long)(h->paired ? h->ntheta / 2 : h->ntheta) * K;  // paired: one lane group per pair
    const long warps = ((samples + (32 / LPS) - 1) / (32 / LPS)) * (h->zs / (LPS * ZV));
    const long blocks = (warps * 32 + kThreads - 1) / kThreads;
    const float scale = (float)(1.0 / (4.0 * h->n * (double)h->n));
#define MM_G(MM)                                                                                          \
    case MM:                                                                                              \
        if (h->paired)                                                                                    \
            k_gather_pair<ZV, LPS, MM, ZSC><<<blocks, kThreads, 0, st>>>(h->F, h->Hh, h->d_cos, h->d_sin, h->n, \
                                                                    h->ntheta, h->zs, h->c0, h->c1, scale, \
                                                                    h->clamp);                              \
        else                                                                                              \
            k_gather<ZV, LPS, MM, ZSC><<<blocks, kThreads, 0, st>>>(h->F, h->Hh, h->d_cos, h->d_sin, h->n, \
                                                               h->ntheta, h->zs, h->c0, h->c1, scale,      \
                                                               h->clamp);                                  \
        break;
    switch (h->m) {
        MM_G(2) MM_G(3) MM_G(4) MM_G(5) MM_G(6)
        default: MM_REQUIRE(false, "unsupported m=%d", h->m);
    }
#undef MM_G
    MM_LAUNCHED();
    return MM_OK;
}

int launch_gather(mm_tomo* h, cudaStream_t st) {
    int ZV, LPS;
    pick_lanes(h->zs, ZV, LPS);
    if (ZV == 1) return launch_gather_m<1, 1, 0>(h, st);
    switch (LPS) {
        case 1: return launch_gather_m<2, 1, 0>(h, st);
        case 2: return launch_gather_m<2, 2, 0>(h, st);
        case 4: return launch_gather_m<2, 4, 0>(h, st);
        case 8: return launch_gather_m<2, 8, 0>(h, st);
        case 16: return launch_gather_m<2, 16, 0>(h, st);
        default:  // 64 slices (the production slab) with compile-time tap offsets
            return h->zs == 64 ? launch_gather_m<2, 32, 64>(h, st) : launch_gather_m<2, 32, 0>(h, st);
    }
}

int ensure_rt(mm_tomo* h, cudaStream_t st) {
    if (!h->plans_rt) {
        const int n = h->n, T = h->ntheta, zs = h->zs;
        size_t ws = h->fft_work_bytes;
        if (!h->fused_r)
            MM_TRY(plan1d(&h->plan_rr2c, n, 1, n, (long long)T * zs, 1, CUFFT_R2C, (long long)T * zs, &ws));
        if (!h->fused_x)
            MM_TRY(plan1d(&h->plan_xc2r, 2 * n, 1, n + 1, 1, 2 * n, CUFFT_C2R, (long long)zs * n, &ws));
        h->plans_rt = true;
        MM_TRY(ensure_work(h, ws));
    }
    return mmtomo::build_csr(h, st);
}

void destroy(mm_tomo* h) {
    h->tm.release();
    mmtomo::free_tables(h);
    cufftHandle all[6] = {h->plan_xr2c, h->plan_xc2r, h->plan_y, h->plan_rc2r, h->plan_rr2c, h->plan_rc2c};
    for (cufftHandle p : all)
        if (p) cufftDestroy(p);
    void* bufs[] = {h->d_cos, h->d_sin, h->d_phi1, h->d_twy, h->d_tww, h->d_twr, h->d_exr, h->col_scratch, h->col_tw, h->P, h->X, h->Y, h->F, h->Hh, h->sino_tmp, h->fft_work,
                    h->ypad, h->yc};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete h;
}

}  // namespace

// ==========================================================================
extern "C" int mm_tomo_create(int n, int nz, int ntheta, const float* theta_host, const mm_tomo_opts* opts,
                              mm_tomo** out) {
    MM_REQUIRE(out != nullptr, "mm_tomo_create: out is NULL");
    *out = nullptr;
    MM_REQUIRE(n >= 8 && n <= 32768 && n % 2 == 0, "mm_tomo_create: n=%d must be even and in [8, 32768]", n);
    MM_REQUIRE(nz >= 1 && nz <= 4096, "mm_tomo_create: nz=%d out of range", nz);
    MM_REQUIRE(ntheta >= 1 && theta_host != nullptr, "mm_tomo_create: need ntheta >= 1 angles");
    const double eps = (opts && opts->eps > 0) ? opts->eps : 1e-3;
    const double mu = -log(eps) / (2.0 * n * n);
    int m = (int)ceil(2.0 * n / M_PI * sqrt(-mu * log(eps) + (mu * n) * (mu * n) / 4.0));
    if (opts && opts->m > 0) m = opts->m;
    MM_REQUIRE(!opts || opts->max_table_angles >= 0, "mm_tomo_create: max_table_angles must be >= 0");
    MM_REQUIRE(m >= 2 && m <= 6, "mm_tomo_create: m=%d unsupported (2..6)", m);

    mm_tomo* h = new mm_tomo();
    h->n = n;
    h->nz = nz;
    h->ntheta = ntheta;
    h->m = m;
    h->K = n / 2 + 1;
    h->clamp = (opts && opts->clamp_xy) ? 1 : 0;
    h->compensated = (opts && opts->compensated) ? 1 : 0;
    h->table_angles = opts ? opts->max_table_angles : 0;
    int zs = 1;
    while (zs < nz) zs <<= 1;
    h->zs = zs;
    h->mu = (float)mu;  // the reference hands mu to its kernels as float32
    h->c0 = 3.141592653589793238f / h->mu;
    h->c1 = -3.141592653589793238f * 3.141592653589793238f / h->mu;
    h->phi_scale = (float)((double)(1 - n % 4) / (n * sqrt((double)n * ntheta)));
    cudaGetDevice(&h->device);
    cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);

    auto fail = [&](int rc) {
        destroy(h);
        return rc;
    };
    int rc;
    std::vector<float> cs(ntheta), sn(ntheta), ph(n);
    if (ntheta % 2 == 0) {
        bool sym = true;
        for (int t = 0; t < ntheta / 2 && sym; ++t) {
            const double d = fmod((double)theta_host[t + ntheta / 2] - (double)theta_host[t] + 4.0 * M_PI, 2.0 * M_PI);
            sym = fabs(d - M_PI) < 1e-4;
        }
        h->paired = sym ? 1 : 0;
    }
    for (int t = 0; t < ntheta; ++t) {
        cs[t] = (float)cos((double)theta_host[t]);
        sn[t] = (float)sin((double)theta_host[t]);
    }
    for (int i = 0; i < n; ++i) {
        const float tf = (float)(-0.5 + (double)i / n);   // linspace(-1/2, 1/2, n) in float32
        const double td = tf;
        ph[i] = (float)exp(mu * (double)n * n * td * td);
    }
    if ((rc = alloc(h, &h->d_cos, ntheta, "cos table")) || (rc = alloc(h, &h->d_sin, ntheta, "sin table")) ||
        (rc = alloc(h, &h->d_phi1, n, "phi table")))
        return fail(rc);
    if (native_line(2L * n)) {
        // the table of an L-point line has at most 1.5 L entries; size it 2L
        std::vector<float2> tw(4 * (size_t)n, make_float2(0.f, 0.f));
        stockham::host_twiddles(2 * n, false, tw.data());
        if ((rc = alloc(h, &h->d_twy, tw.size(), "column FFT twiddles"))) return fail(rc);
        if (cudaMemcpy(h->d_twy, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
            mm::set_error("mm_tomo_create: table upload failed");
            return fail(MM_ECUDA);
        }
        if (!mm_is_pow2(2L * n) && 2 * n >= 6144) {  // the wide schedule of the x-side forward and columns
            std::vector<float2> tww(4 * (size_t)n, make_float2(0.f, 0.f));
            stockham::host_twiddles(2 * n, false, tww.data(), true);
            if ((rc = alloc(h, &h->d_tww, tww.size(), "wide column FFT twiddles"))) return fail(rc);
            if (cudaMemcpy(h->d_tww, tww.data(), tww.size() * sizeof(float2), cudaMemcpyHostToDevice) !=
                cudaSuccess) {
                mm::set_error("mm_tomo_create: table upload failed");
                return fail(MM_ECUDA);
            }
        }
        h->fused_x = 2 * n >= 64;
        const int M = n / 2;
        if (M >= 16) {
            std::vector<float2> twr(2 * (size_t)M, make_float2(0.f, 0.f)), exr(M + 1);
            stockham::host_twiddles(M, false, twr.data());
            for (int k = 0; k <= M; ++k) {
                const double a = 2.0 * M_PI * k / n;
                exr[k] = make_float2((float)cos(a), (float)sin(a));
            }
            if ((rc = alloc(h, &h->d_twr, twr.size(), "r FFT twiddles")) ||
                (rc = alloc(h, &h->d_exr, exr.size(), "r packing twiddles")))
                return fail(rc);
            if (cudaMemcpy(h->d_twr, twr.data(), twr.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(h->d_exr, exr.data(), exr.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
                mm::set_error("mm_tomo_create: table upload failed");
                return fail(MM_ECUDA);
            }
            h->fused_r = true;
        }
        if (mmfft::init_constants() != cudaSuccess) {
            mm::set_error("mm_tomo_create: FFT constant upload failed");
            return fail(MM_ECUDA);
        }
        size_t scr = 0, twn = 0;
        if (mmtomo::col_fft_sizes(n, zs, h->sms, &scr, &twn) == MM_OK) {
            std::vector<float2> twc(twn);
            mmtomo::col_fft_twiddles(twc.data());
            if ((rc = alloc(h, &h->col_scratch, scr, "column transform scratch")) ||
                (rc = alloc(h, &h->col_tw, twn, "column transform twiddles")))
                return fail(rc);
            if (cudaMemcpy(h->col_tw, twc.data(), twn * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
                mm::set_error("mm_tomo_create: table upload failed");
                return fail(MM_ECUDA);
            }
        }
    }
    if (cudaMemcpy(h->d_cos, cs.data(), ntheta * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->d_sin, sn.data(), ntheta * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->d_phi1, ph.data(), n * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        mm::set_error("mm_tomo_create: table upload failed");
        return fail(MM_ECUDA);
    }
    const size_t spec = (size_t)2 * n * (n + 1) * zs;
    // P and X serve only the cuFFT x-side (sizes without the fused kernels)
    if (!h->fused_x && ((rc = alloc(h, &h->P, (size_t)zs * n * 2 * n, "padded rows")) ||
                        (rc = alloc(h, &h->X, (size_t)zs * n * (n + 1), "row spectra"))))
        return fail(rc);
    if ((rc = alloc(h, &h->Y, spec, "padded column input")) || (rc = alloc(h, &h->F, spec, "half spectrum")) ||
        (rc = alloc(h, &h->Hh, (size_t)h->K * ntheta * zs, "polar lines")))
        return fail(rc);
    if (cudaMemset(h->Y, 0, spec * sizeof(float2)) != cudaSuccess) {
        mm::set_error("mm_tomo_create: memset failed");
        return fail(MM_ECUDA);
    }
    // cuFFT plans only where no native kernel covers the size
    size_t ws = 0;
    const bool native_col = native_line(2L * n);
    if ((!h->fused_x && (rc = plan1d(&h->plan_xr2c, 2 * n, 1, 2 * n, 1, n + 1, CUFFT_R2C, (long long)zs * n, &ws))) ||
        (!native_col && (rc = plan1d(&h->plan_y, 2 * n, (long long)(n + 1) * zs, 1, (long long)(n + 1) * zs, 1,
                                     CUFFT_C2C, (long long)(n + 1) * zs, &ws))) ||
        (!h->fused_r &&
         (rc = plan1d(&h->plan_rc2r, n, (long long)ntheta * zs, 1, 1, n, CUFFT_C2R, (long long)ntheta * zs, &ws))) ||
        (rc = ensure_work(h, ws)))
        return fail(rc);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        mm::set_error("mm_tomo_create: device error during setup");
        return fail(MM_ECUDA);
    }
    *out = h;
    return MM_OK;
}

extern "C" int mm_tomo_destroy(mm_tomo* h) {
    if (!h) return MM_OK;
    cudaDeviceSynchronize();
    destroy(h);
    return MM_OK;
}

extern "C" size_t mm_tomo_workspace_bytes(const mm_tomo* h) { return h ? h->ws_bytes : 0; }

extern "C" int mm_tomo_R_ex(mm_tomo* h, const void* obj, int obj_dtype, void* sino, int sino_dtype, int nz,
                            void* stream) {
    MM_REQUIRE(h != nullptr, "mm_tomo_R: NULL handle");
    MM_REQUIRE(obj != nullptr && sino != nullptr, "mm_tomo_R: NULL array");
    MM_REQUIRE(nz >= 1 && nz <= h->nz, "mm_tomo_R: nz=%d outside [1, %d]", nz, h->nz);
    MM_REQUIRE((obj_dtype == MM_F32 || obj_dtype == MM_BF16) && (sino_dtype == MM_F32 || sino_dtype == MM_BF16),
               "mm_tomo_R: storage dtypes must be MM_F32 or MM_BF16");
    MM_REQUIRE((obj_dtype == MM_F32 && sino_dtype == MM_F32) || (h->fused_x && h->fused_r && mm_is_pow2(h->n)),
               "mm_tomo_R: bfloat16 storage needs n a power of two in [32, 2048]");
    MM_REQUIRE(((uintptr_t)obj % 4) == 0 && ((uintptr_t)sino % 4) == 0, "mm_tomo_R: misaligned array");
    MM_RANGE(obj, (size_t)nz * h->n * h->n * (obj_dtype == MM_BF16 ? 2 : 4), "mm_tomo_R", "obj");
    MM_RANGE(sino, (size_t)h->ntheta * nz * h->n * (sino_dtype == MM_BF16 ? 2 : 4), "mm_tomo_R", "sino");
    cudaStream_t st = (cudaStream_t)stream;
    const int n = h->n, zs = h->zs, T = h->ntheta;
    h->tm.begin(0, st);
    if (h->y_dirty) {  // rows [0, n/2) and [3n/2, 2n) of Y are the y zero padding
        const size_t half = (size_t)(n / 2) * (n + 1) * zs * sizeof(float2);
        MM_CUDA(cudaMemsetAsync(h->Y, 0, half, st));
        MM_CUDA(cudaMemsetAsync(h->Y + (size_t)(3 * n / 2) * (n + 1) * zs, 0, half, st));
        h->y_dirty = false;
    }
    if (h->fused_x) {  // phi*pad + x real FFT + slice interleave in one pass
        MM_TRY(launch_xfwd(h, obj, obj_dtype, nz, st));
        h->tm.end(st, 1);
    } else {
        k_pad_phi<<<(unsigned)((long)zs * n), kThreads, 0, st>>>((const float*)obj, h->P, h->d_phi1, h->phi_scale,
                                                                 n, nz);
        MM_LAUNCHED();
        h->tm.end(st, 1);
        h->tm.begin(1, st);
        MM_CUFFT(cufftSetStream(h->plan_xr2c, st));
        MM_CUFFT(cufftExecR2C(h->plan_xr2c, h->P, (cufftComplex*)h->X));
        h->tm.end(st, 0);
        h->tm.begin(2, st);
        dim3 tb(32, 8), tg((n + 1 + 31) / 32, (zs + 31) / 32, n);
        k_transpose_in<<<tg, tb, 0, st>>>(h->X, h->Y, n, zs);
        MM_LAUNCHED();
        h->tm.end(st, 1);
    }
    h->tm.begin(3, st);
    int rc = launch_col_fft<false>(h, h->Y, h->F, st);
    if (rc == -100) {
        MM_CUFFT(cufftSetStream(h->plan_y, st));
        MM_CUFFT(cufftExecC2C(h->plan_y, (cufftComplex*)h->Y, (cufftComplex*)h->F, CUFFT_FORWARD));
    } else if (rc != MM_OK) {
        return rc;
    }
    h->tm.end(st, rc == -100 ? 0 : 1);
    h->tm.begin(4, st);
    MM_TRY(launch_gather(h, st));
    h->tm.end(st, 1);
    h->tm.begin(5, st);
    void* dst = sino;
    if (nz < zs) {
        if (!h->sino_tmp) MM_TRY(alloc(h, &h->sino_tmp, (size_t)T * zs * n, "padded sinogram"));
        dst = h->sino_tmp;
    }
    const int dst_dtype = nz < zs ? MM_F32 : sino_dtype;
    if (h->fused_r) {
        MM_TRY(launch_r(h, true, h->Hh, dst, st, dst_dtype));
    } else {
        MM_CUFFT(cufftSetStream(h->plan_rc2r, st));
        MM_CUFFT(cufftExecC2R(h->plan_rc2r, (cufftComplex*)h->Hh, (float*)dst));
    }
    if (nz < zs) {
        if (sino_dtype == MM_BF16)
            k_copy_z_t<float, __nv_bfloat16><<<(unsigned)((long)T * nz), kThreads, 0, st>>>(
                h->sino_tmp, (__nv_bfloat16*)sino, n, zs, nz, nz);
        else
            k_copy_z<<<(unsigned)((long)T * nz), kThreads, 0, st>>>(h->sino_tmp, (float*)sino, n, zs, nz, nz);
        MM_LAUNCHED();
    }
    h->tm.end(st, (nz < zs ? 1 : 0) + (h->fused_r ? 1 : 0));
    return MM_OK;
}

extern "C" int mm_tomo_R(mm_tomo* h, const float* obj, float* sino, int nz, void* stream) {
    return mm_tomo_R_ex(h, obj, MM_F32, sino, MM_F32, nz, stream);
}

extern "C" int mm_tomo_prepare_rt(mm_tomo* h, void* stream) {
    MM_REQUIRE(h != nullptr, "mm_tomo_prepare_rt: NULL handle");
    return ensure_rt(h, (cudaStream_t)stream);
}

namespace {
// scatter + IFFT along v + transposed C2R along x + crop*phi for one real
// run whose line spectra are in Q = h->Hh.  OUT selects the output part.
int rt_tail(mm_tomo* h, cudaStream_t st) {
    const int n = h->n, zs = h->zs;
    h->tm.begin(7, st);
    MM_TRY(mmtomo::launch_scatter(h, h->Hh, h->F, st));
    h->tm.end(st, 0);
    h->tm.begin(8, st);
    int rc = launch_col_fft<true>(h, h->F, h->Y, st);
    if (rc == -100) {
        MM_CUFFT(cufftSetStream(h->plan_y, st));
        MM_CUFFT(cufftExecC2C(h->plan_y, (cufftComplex*)h->F, (cufftComplex*)h->Y, CUFFT_INVERSE));
        h->y_dirty = true;
    } else if (rc != MM_OK) {
        return rc;
    }
    h->tm.end(st, rc == -100 ? 0 : 1);
    if (h->fused_x) return MM_OK;  // the caller's x-side kernel reads Y directly
    h->tm.begin(9, st);
    dim3 tb(32, 8), tg((n + 1 + 31) / 32, (zs + 31) / 32, n);
    k_transpose_out<<<tg, tb, 0, st>>>(h->Y, h->X, n, zs);
    MM_LAUNCHED();
    h->tm.end(st, 1);
    h->tm.begin(10, st);
    MM_CUFFT(cufftSetStream(h->plan_xc2r, st));
    MM_CUFFT(cufftExecC2R(h->plan_xc2r, (cufftComplex*)h->X, h->P));
    h->tm.end(st, 0);
    return MM_OK;
}
}  // namespace

extern "C" int mm_tomo_RT(mm_tomo* h, const void* sino, int dtype, void* obj, int nz, void* stream) {
    MM_REQUIRE(h != nullptr, "mm_tomo_RT: NULL handle");
    MM_REQUIRE(sino != nullptr && obj != nullptr, "mm_tomo_RT: NULL array");
    MM_REQUIRE(dtype == MM_F32 || dtype == MM_C64 || dtype == MM_BF16, "mm_tomo_RT: dtype %d unsupported", dtype);
    MM_REQUIRE(dtype != MM_BF16 || (h->fused_x && h->fused_r && mm_is_pow2(h->n)),
               "mm_tomo_RT: bfloat16 storage needs n a power of two in [32, 2048]");
    MM_REQUIRE(nz >= 1 && nz <= h->nz, "mm_tomo_RT: nz=%d outside [1, %d]", nz, h->nz);
    MM_REQUIRE(((uintptr_t)sino % (dtype == MM_C64 ? 8 : 4)) == 0 && ((uintptr_t)obj % 4) == 0,
               "mm_tomo_RT: misaligned array");
    {
        const size_t esz = dtype == MM_C64 ? 8 : (dtype == MM_BF16 ? 2 : 4);
        MM_RANGE(sino, (size_t)h->ntheta * nz * h->n * esz, "mm_tomo_RT", "sino");
        MM_RANGE(obj, (size_t)nz * h->n * h->n * esz, "mm_tomo_RT", "obj");
    }
    cudaStream_t st = (cudaStream_t)stream;
    MM_TRY(ensure_rt(h, st));
    const int n = h->n, zs = h->zs, T = h->ntheta;
    const unsigned rows = (unsigned)((long)nz * n);
    if (dtype == MM_F32 || dtype == MM_BF16) {
        h->tm.begin(6, st);
        const void* y = sino;
        int ydt = dtype;
        if (nz < zs) {
            if (!h->ypad) MM_TRY(alloc(h, &h->ypad, (size_t)T * zs * n, "padded sinogram"));
            if (dtype == MM_BF16)
                k_copy_z_t<__nv_bfloat16, float><<<(unsigned)((long)T * zs), kThreads, 0, st>>>(
                    (const __nv_bfloat16*)sino, h->ypad, n, nz, zs, nz);
            else
                k_copy_z<<<(unsigned)((long)T * zs), kThreads, 0, st>>>((const float*)sino, h->ypad, n, nz, zs, nz);
            MM_LAUNCHED();
            y = h->ypad;
            ydt = MM_F32;
        }
        if (h->fused_r) {
            MM_TRY(launch_r(h, false, y, h->Hh, st, ydt));
        } else {
            MM_CUFFT(cufftSetStream(h->plan_rr2c, st));
            MM_CUFFT(cufftExecR2C(h->plan_rr2c, (cufftReal*)y, (cufftComplex*)h->Hh));
        }
        h->tm.end(st, (nz < zs ? 1 : 0) + (h->fused_r ? 1 : 0));
        MM_TRY(rt_tail(h, st));
        h->tm.begin(11, st);
        if (h->fused_x) {
            MM_TRY(launch_xinv<0>(h, obj, nz, st, dtype));
        } else {
            k_crop_phi<0><<<rows, kThreads, 0, st>>>(h->P, obj, h->d_phi1, h->phi_scale, n);
            MM_LAUNCHED();
        }
        h->tm.end(st, 1);
        return MM_OK;
    }
    // complex64 sinogram: real and imaginary output parts are two real runs
    if (!h->plans_c) {
        size_t ws = h->fft_work_bytes;
        MM_TRY(plan1d(&h->plan_rc2c, n, 1, n, 1, n, CUFFT_C2C, (long long)T * zs, &ws));
        h->plans_c = true;
        MM_TRY(ensure_work(h, ws));
    }
    if (!h->yc) MM_TRY(alloc(h, &h->yc, (size_t)T * zs * n, "complex line spectra"));
    h->tm.begin(13, st);
    const float2* y = static_cast<const float2*>(sino);
    if (nz < zs) {
        k_copy_z_c<<<(unsigned)((long)T * zs), kThreads, 0, st>>>(y, h->yc, n, nz, zs, nz);
        MM_LAUNCHED();
        y = h->yc;
    }
    MM_CUFFT(cufftSetStream(h->plan_rc2c, st));
    MM_CUFFT(cufftExecC2C(h->plan_rc2c, (cufftComplex*)y, (cufftComplex*)h->yc, CUFFT_FORWARD));
    h->tm.end(st, nz < zs ? 1 : 0);
    for (int part = 0; part < 2; ++part) {
        h->tm.begin(6, st);
        if (part == 0)
            k_combine<0><<<(unsigned)((long)T * zs), kThreads, 0, st>>>(h->yc, h->Hh, n, T, zs);
        else
            k_combine<1><<<(unsigned)((long)T * zs), kThreads, 0, st>>>(h->yc, h->Hh, n, T, zs);
        MM_LAUNCHED();
        h->tm.end(st, 1);
        MM_TRY(rt_tail(h, st));
        h->tm.begin(11, st);
        if (h->fused_x) {
            MM_TRY(part == 0 ? launch_xinv<1>(h, obj, nz, st) : launch_xinv<2>(h, obj, nz, st));
        } else {
            if (part == 0)
                k_crop_phi<1><<<rows, kThreads, 0, st>>>(h->P, obj, h->d_phi1, h->phi_scale, n);
            else
                k_crop_phi<2><<<rows, kThreads, 0, st>>>(h->P, obj, h->d_phi1, h->phi_scale, n);
            MM_LAUNCHED();
        }
        h->tm.end(st, 1);
    }
    return MM_OK;
}

extern "C" int mm_tomo_set_timing(mm_tomo* h, int on) {
    MM_REQUIRE(h != nullptr, "mm_tomo_set_timing: NULL handle");
    h->tm.reset();
    h->tm.on = on != 0;
    return MM_OK;
}

extern "C" int mm_tomo_get_timing(mm_tomo* h, double* ms, long long* calls, int nstages, long long* kernels) {
    MM_REQUIRE(h != nullptr, "mm_tomo_get_timing: NULL handle");
    h->tm.read();
    for (int i = 0; i < nstages && i < mm::StageTimer::kMax; ++i) {
        if (ms) ms[i] = h->tm.ms[i];
        if (calls) calls[i] = h->tm.calls[i];
    }
    if (kernels) *kernels = h->tm.kernels;
    return MM_OK;
}
