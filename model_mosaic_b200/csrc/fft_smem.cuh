// FFTs held in registers, exchanged through shared memory.
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
// W_48^j, for the twiddles of the 24-point register FFT (3 x 8).
static __constant__ float2 c_w48[48];

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
    if (e != cudaSuccess) return e;
    float2 w48[48];
    for (int j = 0; j < 48; ++j) {
        const double a = -2.0 * 3.14159265358979323846 * j / 48.0;
        w48[j] = make_float2((float)cos(a), (float)sin(a));
    }
    e = cudaMemcpyToSymbol(c_w48, w48, sizeof(w48));
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

// W_12^j = exp(-2*pi*i*j/12) as compile-time constants (j folds to a
// constant in unrolled code): the twiddles of the 3 * 2^a register FFTs.
__host__ __device__ constexpr float2 w12(int j) {
    constexpr float h = 0.86602540378443864676f;  // sqrt(3) / 2
    switch (j % 12) {
        case 0: return float2{1.f, 0.f};
        case 1: return float2{h, -0.5f};
        case 2: return float2{0.5f, -h};
        case 3: return float2{0.f, -1.f};
        case 4: return float2{-0.5f, -h};
        case 5: return float2{-h, -0.5f};
        case 6: return float2{-1.f, 0.f};
        case 7: return float2{-h, 0.5f};
        case 8: return float2{-0.5f, h};
        case 9: return float2{0.f, 1.f};
        case 10: return float2{0.5f, h};
        default: return float2{h, 0.5f};
    }
}

template <int R, bool INV>
__device__ __forceinline__ void reg_fft(float2 (&v)[R]);

// In-register FFT of size R = 3M (M = 1, 2, 4): with n = M n1 + n2 and
// k = k1 + 3 k2, a 3-point DFT over n1 for each n2, the twiddle
// W_R^(n2 k1), then an M-point FFT over n2 for each k1.
template <int R, bool INV>
__device__ __forceinline__ void reg_fft3(float2 (&v)[R]) {
    constexpr int M = R / 3;
    constexpr float h = 0.86602540378443864676f;
    constexpr float sh = INV ? -h : h;
    float2 y[3][M];
#pragma unroll
    for (int n2 = 0; n2 < M; ++n2) {
        const float2 a = v[n2], b = v[M + n2], c = v[2 * M + n2];
        const float2 t = make_float2(b.x + c.x, b.y + c.y), d = make_float2(b.x - c.x, b.y - c.y);
        const float2 m = make_float2(a.x - 0.5f * t.x, a.y - 0.5f * t.y);
        y[0][n2] = make_float2(a.x + t.x, a.y + t.y);
        // forward: X1 = m - i h d, X2 = m + i h d (inverse: h -> -h)
        float2 y1 = make_float2(m.x + sh * d.y, m.y - sh * d.x);
        float2 y2 = make_float2(m.x - sh * d.y, m.y + sh * d.x);
        if (n2 > 0) {
            float2 w1, w2;
            if constexpr (12 % R == 0) {  // R = 3, 6, 12: compile-time constants
                w1 = w12(n2 * (12 / R));
                w2 = w12(2 * n2 * (12 / R));
            } else {                      // R = 24: the W_48 table
                static_assert(48 % R == 0, "3 * 2^a register FFTs up to 24 points");
                w1 = c_w48[(n2 * (48 / R)) % 48];
                w2 = c_w48[(2 * n2 * (48 / R)) % 48];
            }
            y1 = INV ? cmulc(y1, w1) : cmul(y1, w1);
            y2 = INV ? cmulc(y2, w2) : cmul(y2, w2);
        }
        y[1][n2] = y1;
        y[2][n2] = y2;
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; ++k1) {
        reg_fft<M, INV>(y[k1]);
#pragma unroll
        for (int k2 = 0; k2 < M; ++k2) v[k1 + 3 * k2] = y[k1][k2];
    }
}

// In-register FFT of size R (a power of two <= 64, or 3, 6, 12, 24), natural
// order in and out.  INV = false: exp(-2 pi i ...); INV = true:
// exp(+2 pi i ...), unnormalised.
template <int R, bool INV>
__device__ __forceinline__ void reg_fft(float2 (&v)[R]) {
    if constexpr (R % 3 == 0) {
        reg_fft3<R, INV>(v);
    } else if constexpr (R > 1) {
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

// ---------------------------------------------------------------------------
// Stockham FFT of one line of length L held in shared memory, L a power of
// two or three times one.
//
// Powers of two: G = L/16 threads cooperate on a line (t in [0, G)), each
// holding V = 16 complex values per pass; pass p has span NS = 16^p and radix
// RP = 16 except the last, RP = L / 16^(P-1).  L = 3 * 2^k: base radix 8 and
// V = 24 values per thread (G = L/24), the last pass of radix 3, 6 or 12
// (L / 8^(P-1)).  In a pass every group j = t + G*q reads x[j + i*L/RP]
// (i < RP), multiplies by W_{NS*RP}^(i*(j mod NS)), does an RP-point
// register FFT and writes y[(j/NS)*NS*RP + (j mod NS) + i*NS]: natural order
// in, natural order out, no bit reversal.  The first pass reads through
// `ld(pos)` and the last writes through `st(pos, value)`, so a transform can
// start from global memory and end in global memory; the passes in between
// use `buf` through the addressing functor `ad(pos)`.  Twiddles: per pass
// p >= 1 a table tw + off_p with W_{NS*RP}^(i*k) at [i*NS + k]; lanes with
// consecutive j read consecutive entries.
namespace stockham {

using mmfft::cmul;
using mmfft::cmulc;
using mmfft::ilog2;
using mmfft::reg_fft;

// Line lengths the engine covers: 2^k and 3 * 2^k.
__host__ __device__ constexpr bool length_ok(long L) {
    return L >= 2 && ((L & (L - 1)) == 0 || (L % 3 == 0 && ((L / 3) & (L / 3 - 1)) == 0));
}

// Schedule of a length-L line: passes of the base radix and one smaller
// radix, the small one last (REV = false) or first (REV = true).  The
// inverse half of a convolution uses the reversed schedule so that its first
// pass owns exactly the elements the forward's last pass produced (see
// conv()).
// VW = 48 selects the wide form of a 3 * 2^k line (L >= 48): base radix 16
// and 48 values per thread, the last pass of radix 3, 6, 12 or 24 -- half the
// threads per line, for kernels that want more lines per block.
template <int L, bool REV = false, int VW = 0>
struct Sched {
    static_assert(length_ok(L), "line length must be 2^k or 3 * 2^k");
    static constexpr bool P2 = (L & (L - 1)) == 0;
    static_assert(VW == 0 || (VW == 48 && !P2 && L >= 48), "wide schedule: 3 * 2^k lines of 48 or more");
    static constexpr bool W = VW == 48;
    static constexpr int B = (P2 || W) ? 16 : 8;                  // base radix
    static constexpr int VB = P2 ? 16 : (W ? 48 : 24);            // values per thread
    static constexpr int K2 = ilog2<P2 ? L : L / 3>();            // exponent of the power-of-two factor
    static constexpr int P = P2 ? (L <= 16 ? 1 : (K2 + 3) / 4) : (W ? 1 + K2 / 4 : 1 + K2 / 3);   // passes
    static constexpr int G = L >= VB ? L / VB : 1;                // threads per line
    static constexpr int V = L >= VB ? VB : L;                    // values per thread
    static constexpr int small = (P2 || W) ? (L >> (4 * (P - 1))) : (L >> (3 * (P - 1)));
    static constexpr int radix(int p) { return REV ? (p == 0 ? small : B) : (p < P - 1 ? B : small); }
    static constexpr int span(int p) {
        int s = 1;
        for (int q = 0; q < p; ++q) s *= radix(q);
        return s;
    }
    static constexpr int tw_off(int p) {  // start of pass p's table
        int o = 0;
        for (int q = 1; q < p; ++q) o += span(q) * radix(q);
        return o;
    }
    static constexpr int tw_size() { return tw_off(P); }
};

// Host-side table for Sched<L, rev, wide ? 48 : 0> (FP64 angles), its tw_size()
// entries: pass p >= 1, W_{NS*RP}^(i*k) at [off_p + i*NS + k].  Returns the
// entry count (at most 1.5 L), or -1 for a length the engine does not cover.
inline int host_twiddles(int L, bool rev, float2* out, bool wide = false) {
    if (!length_ok(L)) return -1;
    const bool p2 = (L & (L - 1)) == 0;
    if (wide && (p2 || L < 48)) return -1;
    int k2 = 0;
    while ((1L << (k2 + 1)) <= (p2 ? L : L / 3)) ++k2;
    const int P = p2 ? (L <= 16 ? 1 : (k2 + 3) / 4) : (wide ? 1 + k2 / 4 : 1 + k2 / 3);
    const int base = (p2 || wide) ? 16 : 8;
    const int small = (p2 || wide) ? (L >> (4 * (P - 1))) : (L >> (3 * (P - 1)));
    auto radix = [&](int p) { return rev ? (p == 0 ? small : base) : (p < P - 1 ? base : small); };
    int o = 0, ns = radix(0);
    for (int p = 1; p < P; ++p) {
        const int rp = radix(p);
        for (int i = 0; i < rp; ++i)
            for (int k = 0; k < ns; ++k) {
                const double a = -2.0 * 3.14159265358979323846 * (double)((long)i * k % (ns * rp)) / (ns * rp);
                out[o + i * ns + k] = make_float2((float)cos(a), (float)sin(a));
            }
        o += ns * rp;
        ns *= rp;
    }
    return o;
}

// Registers of one thread in pass PASS: groups j = t + G*q, element i of
// group j at line position j + i*NG.
template <int L, bool REV, int PASS, int VW = 0>
struct PassShape {
    using S = Sched<L, REV, VW>;
    static constexpr int RP = S::radix(PASS);
    static constexpr int NS = S::span(PASS);
    static constexpr int NG = L / RP;
    static constexpr int Q = NG / S::G;
    static_assert(Q * RP == S::V, "V values per thread in every pass");
};

template <int L, bool REV, int PASS, bool INV, int VW = 0, class Src>
__device__ __forceinline__ void pass_load(
    float2 (&x)[PassShape<L, REV, PASS, VW>::Q][PassShape<L, REV, PASS, VW>::RP], const Src& src, int t,
    const float2* __restrict__ tw) {
    using Sh = PassShape<L, REV, PASS, VW>;
    using S = Sched<L, REV, VW>;
#pragma unroll
    for (int q = 0; q < Sh::Q; ++q) {
        const int j = t + S::G * q;
#pragma unroll
        for (int i = 0; i < Sh::RP; ++i) x[q][i] = src(j + i * Sh::NG);
        if (Sh::NS > 1) {
            const int k = j % Sh::NS;
            const float2* tp = tw + S::tw_off(PASS);
#pragma unroll
            for (int i = 1; i < Sh::RP; ++i) {
                const float2 w = __ldg(tp + i * Sh::NS + k);
                x[q][i] = INV ? cmulc(x[q][i], w) : cmul(x[q][i], w);
            }
        }
        reg_fft<Sh::RP, INV>(x[q]);
    }
}

template <int L, bool REV, int PASS, int VW = 0, class Dst>
__device__ __forceinline__ void pass_store(
    float2 (&x)[PassShape<L, REV, PASS, VW>::Q][PassShape<L, REV, PASS, VW>::RP], const Dst& dst, int t) {
    using Sh = PassShape<L, REV, PASS, VW>;
    using S = Sched<L, REV, VW>;
#pragma unroll
    for (int q = 0; q < Sh::Q; ++q) {
        const int j = t + S::G * q;
        const int k = j % Sh::NS;
        const int base = (j / Sh::NS) * Sh::NS * Sh::RP + k;
#pragma unroll
        for (int i = 0; i < Sh::RP; ++i) dst(base + i * Sh::NS, x[q][i]);
    }
}

// Passes FIRST..LAST of a transform through shared memory; pass 0 reads
// through `ld`, pass P-1 writes through `st`, every other access is buf.
template <int L, bool REV, bool INV, int PASS, int LAST, int VW = 0, class Ld, class St, class Ad>
__device__ __forceinline__ void run(float2* __restrict__ buf, const Ad& ad, const Ld& ld, const St& st, int t,
                                   const float2* __restrict__ tw) {
    using Sh = PassShape<L, REV, PASS, VW>;
    using S = Sched<L, REV, VW>;
    float2 x[Sh::Q][Sh::RP];
    auto from_buf = [&](int pos) -> float2 { return buf[ad(pos)]; };
    if constexpr (PASS == 0) pass_load<L, REV, PASS, INV, VW>(x, ld, t, tw);
    else pass_load<L, REV, PASS, INV, VW>(x, from_buf, t, tw);
    __syncthreads();  // everyone has read this pass's input
    if constexpr (PASS == S::P - 1) {
        pass_store<L, REV, PASS, VW>(x, st, t);
    } else {
        auto to_buf = [&](int pos, float2 v) { buf[ad(pos)] = v; };
        pass_store<L, REV, PASS, VW>(x, to_buf, t);
        __syncthreads();
    }
    if constexpr (PASS < LAST) run<L, REV, INV, PASS + 1, LAST, VW>(buf, ad, ld, st, t, tw);
}

// One transform: natural order in (`ld`) and out (`st`).  Callers
// synchronise before reusing `buf` after it returns.  tw: Sched<L, false, VW>.
template <int L, bool INV, int VW = 0, class Ld, class St, class Ad>
__device__ __forceinline__ void fft(float2* __restrict__ buf, const Ad& ad, const Ld& ld, const St& st, int t,
                                    const float2* __restrict__ tw) {
    run<L, false, INV, 0, Sched<L, false, VW>::P - 1, VW>(buf, ad, ld, st, t, tw);
}

// Circular convolution y = IFFT(mul(k) * FFT(x)) (both unnormalised): the
// forward's last pass, the pointwise multiply and the inverse's first pass
// (reversed schedule) run on the same registers.  twf: Sched<L, false>
// table; twi: Sched<L, true> table.  `mul(pos, X)` returns the product for
// spectral index pos.
template <int L, class Ld, class Mul, class St, class Ad>
__device__ __forceinline__ void conv(float2* __restrict__ buf, const Ad& ad, const Ld& ld, const Mul& mul,
                                     const St& st, int t, const float2* __restrict__ twf,
                                     const float2* __restrict__ twi) {
    using F = Sched<L, false>;
    using I = Sched<L, true>;
    constexpr int P = F::P;
    if constexpr (P == 1) {
        using Sh = PassShape<L, false, 0>;
        float2 x[Sh::Q][Sh::RP];
        pass_load<L, false, 0, false>(x, ld, t, twf);
#pragma unroll
        for (int q = 0; q < Sh::Q; ++q) {
#pragma unroll
            for (int i = 0; i < Sh::RP; ++i) x[q][i] = mul((t + F::G * q) + i * Sh::NG, x[q][i]);
            reg_fft<Sh::RP, true>(x[q]);
        }
        __syncthreads();
        pass_store<L, false, 0>(x, st, t);
    } else {
        auto to_buf = [&](int pos, float2 v) { buf[ad(pos)] = v; };
        auto from_buf = [&](int pos) -> float2 { return buf[ad(pos)]; };
        run<L, false, false, 0, P - 2>(buf, ad, ld, to_buf, t, twf);
        using Sf = PassShape<L, false, P - 1>;
        using Si = PassShape<L, true, 0>;
        static_assert(Sf::RP == Si::RP && Sf::NG == Si::NG && Sf::Q == Si::Q, "fused pass shapes");
        float2 x[Sf::Q][Sf::RP];
        pass_load<L, false, P - 1, false>(x, from_buf, t, twf);
#pragma unroll
        for (int q = 0; q < Sf::Q; ++q) {
            const int j = t + F::G * q;  // forward output k = j + i*NG; inverse input j + i*NG
#pragma unroll
            for (int i = 0; i < Sf::RP; ++i) x[q][i] = mul(j + i * Sf::NG, x[q][i]);
            reg_fft<Sf::RP, true>(x[q]);
        }
        __syncthreads();
        pass_store<L, true, 0>(x, to_buf, t);
        __syncthreads();
        run<L, true, true, 1, P - 1>(buf, ad, ld, st, t, twi);
    }
}

// Pair-coupled convolution y = IFFT(Y) with Y[k] = pair(k, X[k], X[(N-k) mod N])
// and X = FFT(x) (both unnormalised).  The forward's last pass leaves X[k]
// in the registers that the reversed-schedule inverse's first pass consumes;
// the partner X[N-k] is fetched from `buf`, where every thread parks its X
// for one round.  Same tables as conv().
template <int N, class Ld, class Pair, class St, class Ad>
__device__ __forceinline__ void pairconv(float2* __restrict__ buf, const Ad& ad, const Ld& ld, const Pair& pair,
                                         const St& st, int t, const float2* __restrict__ twf,
                                         const float2* __restrict__ twi) {
    using F = Sched<N, false>;
    constexpr int P = F::P;
    using Sf = PassShape<N, false, P - 1>;
    using Si = PassShape<N, true, 0>;
    static_assert(Sf::RP == Si::RP && Sf::NG == Si::NG && Sf::Q == Si::Q, "fused pass shapes");
    auto to_buf = [&](int pos, float2 v) { buf[ad(pos)] = v; };
    auto from_buf = [&](int pos) -> float2 { return buf[ad(pos)]; };
    float2 x[Sf::Q][Sf::RP];
    if constexpr (P == 1) {
        pass_load<N, false, 0, false>(x, ld, t, twf);
    } else {
        run<N, false, false, 0, P - 2>(buf, ad, ld, to_buf, t, twf);
        pass_load<N, false, P - 1, false>(x, from_buf, t, twf);
        __syncthreads();  // everyone has read the last pass's input
    }
#pragma unroll
    for (int q = 0; q < Sf::Q; ++q) {
#pragma unroll
        for (int i = 0; i < Sf::RP; ++i) buf[ad((t + F::G * q) + i * Sf::NG)] = x[q][i];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Sf::Q; ++q) {
        const int j = t + F::G * q;
#pragma unroll
        for (int i = 0; i < Sf::RP; ++i) {
            const int k = j + i * Sf::NG;
            x[q][i] = pair(k, x[q][i], buf[ad(k == 0 ? 0 : N - k)]);
        }
        reg_fft<Sf::RP, true>(x[q]);
    }
    __syncthreads();  // partners read before the inverse overwrites buf
    if constexpr (P == 1) {
        pass_store<N, false, 0>(x, st, t);
    } else {
        pass_store<N, true, 0>(x, to_buf, t);
        __syncthreads();
        run<N, true, true, 1, P - 1>(buf, ad, ld, st, t, twi);
    }
}

// Shared-memory addressing: a row line with one pad slot per 16 entries, or
// column lines interleaved with lanes running over CW columns.
struct RowAddr {
    int base;
    __device__ __forceinline__ int operator()(int pos) const { return base + pos + (pos >> 4); }
};
// With fewer than 16 columns one pad row per 16 keeps the radix-16 pass
// writes (position stride 16) free of bank conflicts.
template <int CW>
struct ColAddr {
    int col;
    __device__ __forceinline__ int operator()(int pos) const {
        return CW >= 16 ? pos * CW + col : (pos + (pos >> 4)) * CW + col;
    }
    static constexpr int rows(int L) { return CW >= 16 ? L : L + L / 16; }
};

}  // namespace stockham
