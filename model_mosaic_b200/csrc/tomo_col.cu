// Column transforms of the USFFT Radon pair: length-2n FFTs along v of the
// slice-interleaved spectrum Y/F[v][u][z] (the rfft2's second axis,
// processing/tomo.py:134-136 forward, :181-182 inverse), for 2n = 4096.
//
// The columns are (u, z) pairs, z fastest, so a row of a group of CW
// adjacent columns is one contiguous CW*8-byte segment.  A shared-memory
// transform can hold only four 4096-point columns per block (32-byte
// segments, two exchange passes): the kernel is then bound by L1 wavefronts,
// one per 32-byte row segment plus the exchanges.  Here a block owns CW = 8
// columns (64-byte segments) and splits the transform as 4096 = 64 x 64
// (row index v = 64 n1 + n2, output k = k1 + 64 k2):
//   step 1: for each n2, a 64-point FFT over n1 held in one thread's
//           registers, times W_4096^(n2 k1), written to y[k1][n2][z];
//   step 2: for each k1, a 64-point FFT over n2 of y[k1][.][z] -> X[k1 + 64 k2].
// The intermediate y of a block (4096 * CW * 8 = 256 KB) is larger than
// shared memory: its first 48 of 64 k1 rows (195 KB) stay in shared memory,
// the other 16 in a 64 KB per-block scratch region of global memory that the
// block rewrites for every column group it takes, so it stays resident in L2
// (about 9.5 MB for all SMs; its stores and loads carry an evict-last policy,
// the streamed spectrum an evict-first one).  The handle owns that scratch.
// With all 512 KB of a 16-column block in L2 scratch (77 MB over 148 SMs), the
// L2 did not hold it: about 1.5 GB per launch of the 2048 x 32-slice profile
// case was written back to DRAM.  The kernel is persistent (one block per SM).
//
// Forward: the input's non-zero rows are the centre rows [1024, 3072) (the y
// zero padding), i.e. n1 in [16, 48); rows beyond radius n + 16 of the
// spectrum origin are not stored (the gather never reads them).
// Inverse: rows beyond that radius are zeros (the scatter leaves them
// unwritten) and are not read; only the centre rows k in [1024, 3072), i.e.
// k2 in [16, 48), are stored (the x-side needs nothing else).
#include "mm_common.cuh"
#include "fft_smem.cuh"
#include "tomo_kernels.cuh"

#include <algorithm>
#include <type_traits>

namespace {

constexpr int L = 4096, R = 64, NTH = 256;

__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ unsigned long long policy_evict_last() {
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
// Loads bypass L1 (.cg): every element is read once per column group, and
// the scratch is rewritten by other threads of the block between reads.
__device__ __forceinline__ float2 ld_hint(const float2* p, unsigned long long pol) {
    float2 v;
    asm volatile("ld.global.cg.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(v.x), "=f"(v.y)
                 : "l"(p), "l"(pol)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_hint(float2* p, float2 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol)
                 : "memory");
}

// twl[n2 * 64 + k1] = W_4096^(n2 * k1) (forward sign), FP64-derived.
// ZSC: the slice count when fixed at compile time (row stride an immediate).
// The intermediate y[k1][n2][z]: rows k1 < KS in shared memory (row stride
// padded by 8 entries so that the four k1 rows a warp reads in step 2 fall in
// alternate half-banks: two wavefronts per 256-byte request), rows k1 >= KS
// in the block's global scratch region.
template <int CW, int KS, bool INV, int ZSC>
__global__ void __launch_bounds__(NTH, 1)
    k_col_l2(const float2* __restrict__ src, float2* __restrict__ dst, float2* __restrict__ scratch,
             const float2* __restrict__ twl, int ngroups, int zs_rt) {
    using off_t = typename std::conditional<(ZSC > 0 && ZSC <= 64), unsigned, long>::type;
    constexpr int n = L / 2, PER = CW * R / NTH;  // 64-point lines per thread per step
    constexpr int GSTRIDE = NTH / CW;             // line index stride between a thread's lines
    constexpr int SROW = R * CW + 8;              // shared row stride (entries)
    static_assert(PER >= 1 && NTH % CW == 0, "block shape");
    extern __shared__ float2 ys[];                // [KS][SROW]
    const int zs = ZSC > 0 ? ZSC : zs_rt;
    const off_t ncols = (off_t)(n + 1) * zs;
    const int z = threadIdx.x % CW, g0 = threadIdx.x / CW;
    float2* __restrict__ yg = scratch + (size_t)blockIdx.x * (R - KS) * R * CW;   // rows KS..63
    const unsigned long long pin = policy_evict_last(), stream = policy_evict_first();

    for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const off_t col0 = (off_t)grp * CW;
        const off_t col = col0 + z;
        const int u = (int)(col0 / zs);
        const int r2max = (n + 16) * (n + 16) - u * u;
        // ---- step 1: lines n2 = g0 + GSTRIDE * f over n1
#pragma unroll 1
        for (int f = 0; f < PER; ++f) {
            const int n2 = g0 + GSTRIDE * f;
            float2 v[R];
#pragma unroll
            for (int n1 = 0; n1 < R; ++n1) {
                const int row = R * n1 + n2;
                bool live;
                if (!INV) {
                    live = n1 >= 16 && n1 < 48;
                } else {
                    const int vw = row < n ? row : row - L;
                    live = vw * vw <= r2max;
                }
                v[n1] = live ? ld_hint(src + (off_t)row * ncols + col, stream) : make_float2(0.f, 0.f);
            }
            mmfft::reg_fft<R, INV>(v);
            const float2* tw = twl + n2 * R;
#pragma unroll
            for (int k1 = 0; k1 < R; ++k1) {
                const float2 w = __ldg(tw + k1);
                const float2 t = INV ? mmfft::cmulc(v[k1], w) : mmfft::cmul(v[k1], w);
                if (k1 < KS) ys[k1 * SROW + n2 * CW + z] = t;
                else st_hint(yg + ((k1 - KS) * R + n2) * CW + z, t, pin);
            }
        }
        __syncthreads();  // the block's y is complete (shared and global writes ordered by the barrier)
        // ---- step 2: lines k1 = g0 + GSTRIDE * f over n2
#pragma unroll 1
        for (int f = 0; f < PER; ++f) {
            const int k1 = g0 + GSTRIDE * f;
            float2 v[R];
            if (k1 < KS) {
#pragma unroll
                for (int n2 = 0; n2 < R; ++n2) v[n2] = ys[k1 * SROW + n2 * CW + z];
            } else {
#pragma unroll
                for (int n2 = 0; n2 < R; ++n2) v[n2] = ld_hint(yg + ((k1 - KS) * R + n2) * CW + z, pin);
            }
            mmfft::reg_fft<R, INV>(v);
#pragma unroll
            for (int k2 = 0; k2 < R; ++k2) {
                const int row = k1 + R * k2;
                bool keep;
                if (INV) {
                    keep = k2 >= 16 && k2 < 48;
                } else {
                    const int vw = row < n ? row : row - L;
                    keep = vw * vw <= r2max;
                }
                if (keep) st_hint(dst + (off_t)row * ncols + col, v[k2], stream);
            }
        }
        __syncthreads();  // y is read before the next group overwrites it
    }
}

constexpr int kCW = 8, kKS = 48;  // columns per block; rows of the intermediate held in shared memory

template <bool INV>
int launch(int zs, const float2* src, float2* dst, float2* scratch, const float2* twl, int blocks, cudaStream_t st) {
    constexpr int n = L / 2;
    const int ngroups = (int)((long)(n + 1) * zs / kCW);
    auto kern = zs == 64 ? k_col_l2<kCW, kKS, INV, 64> : k_col_l2<kCW, kKS, INV, 0>;
    const size_t smem = (size_t)kKS * (R * kCW + 8) * sizeof(float2);
    MM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int grid = std::min(ngroups, blocks);
    kern<<<(unsigned)grid, NTH, smem, st>>>(src, dst, scratch, twl, ngroups, zs);
    MM_LAUNCHED();
    return MM_OK;
}

}  // namespace

namespace mmtomo {

int col_fft_sizes(int n, int zs, int sms, size_t* scratch_elems, size_t* tw_elems) {
    if (2 * n != L || zs % kCW != 0 || sms < 1) return kNotCovered;
    *scratch_elems = (size_t)sms * (R - kKS) * R * kCW;
    *tw_elems = (size_t)R * R;
    return MM_OK;
}

void col_fft_twiddles(float2* tw) {
    for (int a = 0; a < R; ++a)
        for (int b = 0; b < R; ++b) {
            const double ang = -2.0 * 3.14159265358979323846 * (double)((a * b) % L) / L;
            tw[a * R + b] = make_float2((float)cos(ang), (float)sin(ang));
        }
}

int col_fft_pipe(int n, int zs, bool inv, const float2* src, float2* dst, float2* scratch, const float2* twl,
                 int sms, cudaStream_t st) {
    if (2 * n != L || zs % kCW != 0 || !scratch || !twl) return kNotCovered;
    MM_CUDA(mmfft::init_constants());  // this translation unit's copy of the radix-2 constants
    return inv ? launch<true>(zs, src, dst, scratch, twl, sms, st) : launch<false>(zs, src, dst, scratch, twl, sms, st);
}

}  // namespace mmtomo
