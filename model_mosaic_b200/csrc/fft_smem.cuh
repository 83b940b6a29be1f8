// Power-of-two FFTs held in registers, exchanged once through shared memory.
//
// A length L = R1*R2 transform is done in two register steps:
//   x[R2*n1 + n2]  --R1-point FFT over n1, twiddle W_L^(n2*k1)-->  Y[k1][n2]
//   Y[k1][.]       --R2-point FFT over n2-->  X[k1 + R1*k2]
// and the inverse transform of a spectrum held as X[k1 + R1*k2] runs the
// same two steps in the opposite order (R2-point over k2 first), so a
// forward FFT, a pointwise multiply and an inverse FFT cost exactly two
// shared-memory exchanges.  Twiddles inside the register FFTs come from a
// 64-entry constant table (compile-time indices); the inter-step twiddles
// from a per-length table in global memory.  All tables are FP64-derived.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace mmfft {

// W_64^j = exp(-2*pi*i*j/64).  Each translation unit that includes this
// header owns a copy; init_constants() uploads it once per device.
static __constant__ float2 c_w64[64];

static inline cudaError_t init_constants() {
    static bool done[64] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
    float2 w[64];
    for (int j = 0; j < 64; ++j) {
        const double a = -2.0 * 3.14159265358979323846 * j / 64.0;
        w[j] = make_float2((float)cos(a), (float)sin(a));
    }
    e = cudaMemcpyToSymbol(c_w64, w, sizeof(w));
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
    return e;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

template <int R>
__host__ __device__ constexpr int ilog2() {
    return R <= 1 ? 0 : 1 + ilog2<R / 2>();
}

// Bit reversal of i in log2(R) bits, loop-free so that it folds to a
// constant for unrolled indices.
template <int R>
__host__ __device__ constexpr int brev(int i) {
    return (((i & 1) << 5) | ((i & 2) << 3) | ((i & 4) << 1) | ((i & 8) >> 1) | ((i & 16) >> 3) |
            ((i & 32) >> 5)) >> (6 - ilog2<R>());
}

// One radix-2 butterfly layer (span LEN) of an in-register DIT FFT, then the
// next layer; every register index is a compile-time constant.
template <int R, int LEN, bool INV>
__device__ __forceinline__ void dit_layers(float2 (&v)[R]) {
    if constexpr (LEN <= R) {
#pragma unroll
        for (int i = 0; i < R; i += LEN) {
#pragma unroll
            for (int k = 0; k < LEN / 2; ++k) {
                const float2 a = v[i + k];
                float2 b = v[i + k + LEN / 2];
                const int w = k * (64 / LEN);
                if (w == 16) {
                    b = INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
                } else if (w != 0) {
                    b = INV ? cmulc(b, c_w64[w]) : cmul(b, c_w64[w]);
                }
                v[i + k] = make_float2(a.x + b.x, a.y + b.y);
                v[i + k + LEN / 2] = make_float2(a.x - b.x, a.y - b.y);
            }
        }
        dit_layers<R, LEN * 2, INV>(v);
    }
}

// In-register radix-2 FFT of size R <= 64, natural order in and out.
// INV = false: exp(-2 pi i ...); INV = true: exp(+2 pi i ...), unnormalised.
template <int R, bool INV>
__device__ __forceinline__ void reg_fft(float2 (&v)[R]) {
    if constexpr (R > 1) {
        float2 t[R];
#pragma unroll
        for (int i = 0; i < R; ++i) t[i] = v[brev<R>(i)];
        dit_layers<R, 2, INV>(t);
#pragma unroll
        for (int i = 0; i < R; ++i) v[i] = t[i];
    }
}

// Factorisation L = R1 * R2 with R1 >= R2 used by the kernels.
template <int L>
struct Split;
template <> struct Split<4> { static constexpr int R1 = 2, R2 = 2; };
template <> struct Split<8> { static constexpr int R1 = 4, R2 = 2; };
template <> struct Split<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Split<32> { static constexpr int R1 = 8, R2 = 4; };
template <> struct Split<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Split<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct Split<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Split<512> { static constexpr int R1 = 32, R2 = 16; };
template <> struct Split<1024> { static constexpr int R1 = 32, R2 = 32; };
template <> struct Split<2048> { static constexpr int R1 = 64, R2 = 32; };
template <> struct Split<4096> { static constexpr int R1 = 64, R2 = 64; };

}  // namespace mmfft
