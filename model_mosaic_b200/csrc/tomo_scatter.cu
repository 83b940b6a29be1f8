// Adjoint of the USFFT gather (TomoReal.RT's scatter, processing/kernels.py:16-93
// with dir = 1): a deterministic pull over a static table built once per
// handle (destination cell pair -> (sample, weights, conj bits)), no atomics.
#include "tomo_int.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

using mm::dev_alloc;

namespace {

// One term w*v of a scatter sum; KAHAN keeps a running compensation c of the
// rounding error of each addition (Kahan 1965), the rest is a plain FMA.
template <bool KAHAN>
__device__ __forceinline__ void acc_add(float& s, float& c, float w, float v) {
    if constexpr (KAHAN) {
        const float y = fmaf(w, v, -c);
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    } else {
        s = fmaf(w, v, s);
    }
}

constexpr unsigned kChunk = 256;  // longest list one lane group sums alone

// Sums of the table entries [e0, e1) of one cell pair, left cell in al
// (compensation cl), right cell in ar (cr).
template <int ZV, int LPS, bool KAHAN>
__device__ __forceinline__ void pair_sums(unsigned e0, unsigned e1, const unsigned* __restrict__ idx,
                                          const float2* __restrict__ wgt, const float2* __restrict__ Q, int zs,
                                          int zoff, int lane, float* al, float* cl, float* ar, float* cr) {
    auto add = [&](unsigned ii, float2 w, const float* v) {
        const float sl = (ii >> 31) ? -w.x : w.x, sr = ((ii >> 30) & 1u) ? -w.y : w.y;
#pragma unroll
        for (int q = 0; q < 2 * ZV; q += 2) {
            acc_add<KAHAN>(al[q], cl[q], w.x, v[q]);
            acc_add<KAHAN>(al[q + 1], cl[q + 1], sl, v[q + 1]);
            acc_add<KAHAN>(ar[q], cr[q], w.y, v[q]);
            acc_add<KAHAN>(ar[q + 1], cr[q + 1], sr, v[q + 1]);
        }
    };
    if constexpr (LPS == 32) {
        // one pair per warp: 32 table entries per coalesced load, handed out
        // by shuffles, four independent spectrum loads in flight
        const unsigned FULL = 0xffffffffu;
        for (unsigned base = e0; base < e1; base += 32) {
            const int cnt = (int)min(32u, e1 - base);
            unsigned mi = 0;
            float2 mw = make_float2(0.f, 0.f);
            if (lane < cnt) {
                mi = __ldg(idx + base + lane);
                mw = __ldg(wgt + base + lane);
            }
            int k = 0;
            for (; k + 4 <= cnt; k += 4) {
                unsigned ii[4];
                float2 ww[4];
                float vv[4][2 * ZV];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    ii[u] = __shfl_sync(FULL, mi, k + u);
                    ww[u].x = __shfl_sync(FULL, mw.x, k + u);
                    ww[u].y = __shfl_sync(FULL, mw.y, k + u);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) ZVec<ZV>::load(Q + (long)(ii[u] & 0x3fffffffu) * zs + zoff, vv[u]);
#pragma unroll
                for (int u = 0; u < 4; ++u) add(ii[u], ww[u], vv[u]);
            }
            for (; k < cnt; ++k) {
                const unsigned ia = __shfl_sync(FULL, mi, k);
                float2 wa;
                wa.x = __shfl_sync(FULL, mw.x, k);
                wa.y = __shfl_sync(FULL, mw.y, k);
                float va[2 * ZV];
                ZVec<ZV>::load(Q + (long)(ia & 0x3fffffffu) * zs + zoff, va);
                add(ia, wa, va);
            }
        }
    } else {
        unsigned e = e0;
        for (; e + 2 <= e1; e += 2) {
            const unsigned ia = __ldg(idx + e), ib = __ldg(idx + e + 1);
            const float2 wa = __ldg(wgt + e), wb = __ldg(wgt + e + 1);
            float va[2 * ZV], vb[2 * ZV];
            ZVec<ZV>::load(Q + (long)(ia & 0x3fffffffu) * zs + zoff, va);
            ZVec<ZV>::load(Q + (long)(ib & 0x3fffffffu) * zs + zoff, vb);
            add(ia, wa, va);
            add(ib, wb, vb);
        }
        if (e < e1) {
            const unsigned ia = __ldg(idx + e);
            const float2 wa = __ldg(wgt + e);
            float va[2 * ZV];
            ZVec<ZV>::load(Q + (long)(ia & 0x3fffffffu) * zs + zoff, va);
            add(ia, wa, va);
        }
    }
}

// Destination cells of pair p; cells beyond radius n + 16 receive nothing
// and with `prune` are not written (k_col_fft reads them as zeros).
struct PairCells {
    long cell;
    bool keepL, keepR;
    __device__ __forceinline__ PairCells(long p, int n, int prune) {
        const int NP = n / 2 + 1;
        const int row = (int)(p / NP), c0 = (int)(p % NP) * 2;
        const int vw = row < n ? row : row - 2 * n;
        const int lim = (n + 16) * (n + 16) - vw * vw;
        keepL = !prune || c0 * c0 <= lim;
        keepR = c0 + 1 <= n && (!prune || (c0 + 1) * (c0 + 1) <= lim);
        cell = (long)row * (n + 1) + c0;
    }
};

// One lane group per (pair or piece, slice group): the warp decomposition
// shared by the three scatter kernels.
template <int ZV, int LPS>
struct ScatterLanes {
    int lane, zoff;
    long item;
    __device__ __forceinline__ ScatterLanes(int zs) {
        constexpr int SPW = 32 / LPS;
        lane = threadIdx.x & 31;
        const int sub = lane / LPS, zl = lane % LPS;
        const int zgroups = zs / (LPS * ZV);
        const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        item = (warp / zgroups) * SPW + sub;
        zoff = (int)(warp % zgroups) * (LPS * ZV) + zl * ZV;
    }
};

// Store (acc = 0) or add (acc != 0: a later block of angles) the sums of a
// cell pair.  Each cell belongs to exactly one lane group per launch.
template <int ZV>
__device__ __forceinline__ void store_cells(float2* __restrict__ A, const PairCells& pc, int zs, int zoff, float* al,
                                            float* ar, int acc) {
    if (pc.keepL) {
        float2* d = A + pc.cell * zs + zoff;
        if (acc) {
            float o[2 * ZV];
            ZVec<ZV>::load(d, o);
#pragma unroll
            for (int q = 0; q < 2 * ZV; ++q) al[q] += o[q];
        }
        ZVec<ZV>::store(d, al);
    }
    if (pc.keepR) {
        float2* d = A + (pc.cell + 1) * zs + zoff;
        if (acc) {
            float o[2 * ZV];
            ZVec<ZV>::load(d, o);
#pragma unroll
            for (int q = 0; q < 2 * ZV; ++q) ar[q] += o[q];
        }
        ZVec<ZV>::store(d, ar);
    }
}

// RT: pull-scatter over the static pair table.  One lane group per pair of
// horizontally adjacent cells (row, 2p) and (row, 2p+1): the two cells
// receive almost the same samples (8 of a window's 9 columns cover both), so
// each table entry carries the sample's weight for either cell and the
// sample's spectrum row is loaded once for both.  idx bit 31 / bit 30:
// conjugate for the left / right cell.  Pairs with more than kChunk entries
// are left to k_scatter_pieces / k_scatter_combine.
template <int ZV, int LPS, bool KAHAN, int ZSC>
__global__ void __launch_bounds__(kThreads) k_scatter(const unsigned* __restrict__ ptr,
                                                      const unsigned* __restrict__ idx,
                                                      const float2* __restrict__ wgt,
                                                      const float2* __restrict__ Q, float2* __restrict__ A,
                                                      long npairs, int zs_rt, int n, int prune, int acc) {
    const int zs = ZSC > 0 ? ZSC : zs_rt;  // compile-time slice count: immediate offsets
    const ScatterLanes<ZV, LPS> ln(zs);
    const long p = ln.item;
    if (p >= npairs) return;
    const PairCells pc(p, n, prune);
    if (!pc.keepL && !pc.keepR) return;
    const unsigned e0 = __ldg(ptr + p), e1 = __ldg(ptr + p + 1);
    if (e1 - e0 > kChunk) return;
    if (acc && e1 == e0) return;
    float al[2 * ZV], cl[2 * ZV], ar[2 * ZV], cr[2 * ZV];
#pragma unroll
    for (int q = 0; q < 2 * ZV; ++q) al[q] = cl[q] = ar[q] = cr[q] = 0.f;
    pair_sums<ZV, LPS, KAHAN>(e0, e1, idx, wgt, Q, zs, ln.zoff, ln.lane, al, cl, ar, cr);
    store_cells<ZV>(A, pc, zs, ln.zoff, al, ar, acc);
}

// Pieces of the long lists: partial sums of kChunk entries each.  With
// KAHAN the partial is the compensated sum s - c.
template <int ZV, int LPS, bool KAHAN, int ZSC>
__global__ void __launch_bounds__(kThreads) k_scatter_pieces(const uint2* __restrict__ task,
                                                             const unsigned* __restrict__ idx,
                                                             const float2* __restrict__ wgt,
                                                             const float2* __restrict__ Q,
                                                             float2* __restrict__ part, long ntasks, int zs_rt) {
    const int zs = ZSC > 0 ? ZSC : zs_rt;
    const ScatterLanes<ZV, LPS> ln(zs);
    if (ln.item >= ntasks) return;
    const uint2 tk = __ldg(task + ln.item);
    float al[2 * ZV], cl[2 * ZV], ar[2 * ZV], cr[2 * ZV];
#pragma unroll
    for (int q = 0; q < 2 * ZV; ++q) al[q] = cl[q] = ar[q] = cr[q] = 0.f;
    pair_sums<ZV, LPS, KAHAN>(tk.x, tk.y, idx, wgt, Q, zs, ln.zoff, ln.lane, al, cl, ar, cr);
    if constexpr (KAHAN) {
#pragma unroll
        for (int q = 0; q < 2 * ZV; ++q) {
            al[q] -= cl[q];
            ar[q] -= cr[q];
        }
    }
    ZVec<ZV>::store(part + (2 * ln.item) * zs + ln.zoff, al);
    ZVec<ZV>::store(part + (2 * ln.item + 1) * zs + ln.zoff, ar);
}

// Long pairs: their pieces' partial sums added in piece order.
template <int ZV, int LPS, bool KAHAN, int ZSC>
__global__ void __launch_bounds__(kThreads) k_scatter_combine(const uint4* __restrict__ lp,
                                                              const float2* __restrict__ part,
                                                              float2* __restrict__ A, long nlong, int zs_rt, int n,
                                                              int prune, int acc) {
    const int zs = ZSC > 0 ? ZSC : zs_rt;
    const ScatterLanes<ZV, LPS> ln(zs);
    if (ln.item >= nlong) return;
    const uint4 q4 = __ldg(lp + ln.item);
    const PairCells pc((long)q4.x, n, prune);
    if (!pc.keepL && !pc.keepR) return;
    float al[2 * ZV], cl[2 * ZV], ar[2 * ZV], cr[2 * ZV];
#pragma unroll
    for (int q = 0; q < 2 * ZV; ++q) al[q] = cl[q] = ar[q] = cr[q] = 0.f;
    for (unsigned t = q4.y; t < q4.z; ++t) {
        float vl[2 * ZV], vr[2 * ZV];
        ZVec<ZV>::load(part + (2L * t) * zs + ln.zoff, vl);
        ZVec<ZV>::load(part + (2L * t + 1) * zs + ln.zoff, vr);
#pragma unroll
        for (int q = 0; q < 2 * ZV; ++q) {
            acc_add<KAHAN>(al[q], cl[q], 1.0f, vl[q]);
            acc_add<KAHAN>(ar[q], cr[q], 1.0f, vr[q]);
        }
    }
    store_cells<ZV>(A, pc, zs, ln.zoff, al, ar, acc);
}

// Scatter-table construction ---------------------------------------------
// Every tap e = (sample s, tap) of every polar sample gets the key
//   (pair << 33) | (e << 1) | half,  pair = row * (n/2+1) + col/2, half = col & 1,
// for its destination cell (row, col); sorted, the taps of one cell pair come
// in sample order, and a left-cell tap followed by the same sample's
// right-cell tap merges into one entry.
template <int M>
__device__ __forceinline__ void tap_dest(long e, int n, int T, const float* __restrict__ cosT,
                                         const float* __restrict__ sinT, SampleGeo& g, int& k, int& t, int& i0,
                                         int& i1, int& row, int& col, bool& cj) {
    constexpr int L = 2 * M + 1;
    const int K = n / 2 + 1;
    const long s = e / (L * L);
    const int tap = (int)(e % (L * L));
    t = (int)(s / K);
    k = (int)(s % K);
    g = sample_geo(t, k, n, M, cosT, sinT);
    i0 = tap % L;
    i1 = tap / L;
    tap_cell(g.bx + i0, g.by + i1, n, row, col, cj);
}

// A table block covers the taps e0 .. e0 + nent - 1 (whole angles); keys
// carry the tap's offset e - e0 within the block.
template <int M>
__global__ void k_pair_keys(unsigned long long* __restrict__ keys, const float* __restrict__ cosT,
                            const float* __restrict__ sinT, int n, int T, long nent, long e0) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nent) return;
    SampleGeo g;
    int k, t, i0, i1, row, col;
    bool cj;
    tap_dest<M>(e0 + e, n, T, cosT, sinT, g, k, t, i0, i1, row, col, cj);
    const unsigned long long pair = (unsigned long long)row * (n / 2 + 1) + (col >> 1);
    keys[e] = (pair << 33) | ((unsigned long long)e << 1) | (unsigned long long)(col & 1);
}

// head[i] = 0 when sorted tap i is the right half merged into tap i-1.
template <int M>
__global__ void k_pair_heads(const unsigned long long* __restrict__ keys, unsigned* __restrict__ head, long nent) {
    constexpr int LL = (2 * M + 1) * (2 * M + 1);
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nent) return;
    unsigned h = 1;
    if (i > 0) {
        const unsigned long long a = keys[i - 1], b = keys[i];
        const bool same_pair = (a >> 33) == (b >> 33);
        const bool same_sample = ((a >> 1) & 0xffffffffull) / LL == ((b >> 1) & 0xffffffffull) / LL;
        if (same_pair && same_sample && (a & 1) == 0 && (b & 1) == 1) h = 0;
    }
    head[i] = h;
}

template <int M>
__device__ __forceinline__ float tap_wgt(const SampleGeo& g, int k, int i0, int i1, int n, float c0, float c1,
                                         float scale) {
    const float inv_twon = 1.0f / (float)(2 * n);
    const float wx = tap_weight(g.bx + i0, g.x0, inv_twon, c1);
    const float wy = c0 * tap_weight(g.by + i1, g.y0, inv_twon, c1);
    // transpose of H = (-1)^j g / (4n^2) followed by the C2R along r, which
    // counts the interior bins twice
    const float ck = (k > 0 && k < n / 2) ? 2.f : 1.f;
    const float sj = (g.j & 1) ? -1.f : 1.f;
    return (wy * wx) * (ck * sj * scale);
}

// Compacted entry of every head: sample index (k*T + t) with the two conj
// bits, (left, right) weights, and its pair for the row pointers.
template <int M>
__global__ void k_pair_payload(const unsigned long long* __restrict__ keys, const unsigned* __restrict__ head,
                               const unsigned* __restrict__ pos, unsigned* __restrict__ idx,
                               float2* __restrict__ wgt, unsigned* __restrict__ pairs,
                               const float* __restrict__ cosT, const float* __restrict__ sinT, int n, int T,
                               long nent, long e0, float c0, float c1, float scale) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nent || !head[i]) return;
    const bool merged = i + 1 < nent && !head[i + 1];
    float w[2] = {0.f, 0.f};
    unsigned conj = 0, sidx = 0;
    for (long j = i; j <= (merged ? i + 1 : i); ++j) {
        const unsigned long long key = keys[j];
        SampleGeo g;
        int k, t, i0, i1, row, col;
        bool cj;
        tap_dest<M>(e0 + (long)((key >> 1) & 0xffffffffull), n, T, cosT, sinT, g, k, t, i0, i1, row, col, cj);
        const int half = (int)(key & 1);
        w[half] = tap_wgt<M>(g, k, i0, i1, n, c0, c1, scale);
        if (cj != g.mir) conj |= half ? 0x40000000u : 0x80000000u;
        sidx = (unsigned)((long)k * T + t);
    }
    const unsigned o = pos[i];
    idx[o] = sidx | conj;
    wgt[o] = make_float2(w[0], w[1]);
    pairs[o] = (unsigned)(keys[i] >> 33);
}

// ptr[p] = first entry of pair p (entries sorted by pair).
__global__ void k_pair_ptr(const unsigned* __restrict__ pairs, unsigned* __restrict__ ptr, long nnz, long npairs) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nnz) return;
    const long prev = (i == 0) ? -1 : (long)pairs[i - 1];
    const long cur = (i == nnz) ? npairs : (long)pairs[i];
    for (long c = prev + 1; c <= cur; ++c) ptr[c] = (unsigned)i;
}

template <int ZV, int LPS>
int launch_scatter_t(mm_tomo* h, const ScatterTable& tb, const float2* Q, float2* A, int acc, cudaStream_t st) {
    const long npairs = 2L * h->n * (h->n / 2 + 1);
    const long warps = ((npairs + (32 / LPS) - 1) / (32 / LPS)) * (h->zs / (LPS * ZV));
    const long blocks = (warps * 32 + kThreads - 1) / kThreads;
    constexpr int Z64 = (ZV == 2 && LPS == 32) ? 64 : 0;  // the production slab: compile-time tap offsets
    const bool z64 = Z64 > 0 && h->zs == 64, kh = h->compensated != 0;
    auto kern = kh ? (z64 ? k_scatter<ZV, LPS, true, Z64> : k_scatter<ZV, LPS, true, 0>)
                   : (z64 ? k_scatter<ZV, LPS, false, Z64> : k_scatter<ZV, LPS, false, 0>);
    // the native inverse column transform treats cells beyond radius n + 16
    // as zeros; cuFFT (other sizes) reads them, so they are written then
    const int L = 2 * h->n;
    const int prune = native_line(L) ? 1 : 0;
    auto grid = [&](long items) {
        const long w = ((items + (32 / LPS) - 1) / (32 / LPS)) * (h->zs / (LPS * ZV));
        return (unsigned)((w * 32 + kThreads - 1) / kThreads);
    };
    if (tb.nchunks > 0) {  // the long lists' pieces first: they are the longest chains
        auto kp = kh ? (z64 ? k_scatter_pieces<ZV, LPS, true, Z64> : k_scatter_pieces<ZV, LPS, true, 0>)
                     : (z64 ? k_scatter_pieces<ZV, LPS, false, Z64> : k_scatter_pieces<ZV, LPS, false, 0>);
        kp<<<grid(tb.nchunks), kThreads, 0, st>>>(tb.chunk_task, tb.idx, tb.w, Q, tb.chunk_part, tb.nchunks, h->zs);
        MM_LAUNCHED();
    }
    kern<<<blocks, kThreads, 0, st>>>(tb.ptr, tb.idx, tb.w, Q, A, npairs, h->zs, h->n, prune, acc);
    MM_LAUNCHED();
    if (tb.nlong > 0) {
        auto kc = kh ? (z64 ? k_scatter_combine<ZV, LPS, true, Z64> : k_scatter_combine<ZV, LPS, true, 0>)
                     : (z64 ? k_scatter_combine<ZV, LPS, false, Z64> : k_scatter_combine<ZV, LPS, false, 0>);
        kc<<<grid(tb.nlong), kThreads, 0, st>>>(tb.chunk_pair, tb.chunk_part, A, tb.nlong, h->zs, h->n, prune, acc);
        MM_LAUNCHED();
    }
    return MM_OK;
}

int launch_table(mm_tomo* h, const ScatterTable& tb, const float2* Q, float2* A, int acc, cudaStream_t st) {
    int ZV, LPS;
    pick_lanes(h->zs, ZV, LPS);
    if (ZV == 1) return launch_scatter_t<1, 1>(h, tb, Q, A, acc, st);
    switch (LPS) {
        case 1: return launch_scatter_t<2, 1>(h, tb, Q, A, acc, st);
        case 2: return launch_scatter_t<2, 2>(h, tb, Q, A, acc, st);
        case 4: return launch_scatter_t<2, 4>(h, tb, Q, A, acc, st);
        case 8: return launch_scatter_t<2, 8>(h, tb, Q, A, acc, st);
        case 16: return launch_scatter_t<2, 16>(h, tb, Q, A, acc, st);
        default: return launch_scatter_t<2, 32>(h, tb, Q, A, acc, st);
    }
}

void free_table(mm_tomo* h, ScatterTable& tb) {
    void* bufs[] = {tb.ptr, tb.idx, tb.w, tb.chunk_task, tb.chunk_pair, tb.chunk_part};
    for (void* b : bufs)
        if (b) cudaFree(b);
    h->ws_bytes -= tb.bytes;
    const int t0 = tb.t0, t1 = tb.t1;
    tb = ScatterTable();
    tb.t0 = t0;
    tb.t1 = t1;
}

template <typename Tp>
int talloc(mm_tomo* h, ScatterTable& tb, Tp** p, size_t count, const char* what) {
    MM_TRY(alloc(h, p, count, what));
    tb.bytes += count * sizeof(Tp);
    return MM_OK;
}

constexpr int kBuildBytesPerTap = 26;  // keys (2 x 8), merge flags, positions, sort/scan temp

// Builds the table of the angles [tb.t0, tb.t1): every tap of every sample
// gets the key (pair << 33) | (tap offset in the block << 1) | half for its
// destination cell; sorted, the taps of one cell pair come in sample order
// and a left-cell tap followed by the same sample's right-cell tap merges
// into one entry.
int build_table(mm_tomo* h, ScatterTable& tb, cudaStream_t st) {
    const int n = h->n, T = h->ntheta, M = h->m, L = 2 * M + 1;
    const long per_angle = (long)h->K * L * L;
    const long nent = (long)(tb.t1 - tb.t0) * per_angle, e0 = (long)tb.t0 * per_angle;
    const long npairs = 2L * n * (n / 2 + 1);
    MM_REQUIRE(nent < (1L << 32) && (long)T * h->K < (1L << 30), "adjoint table too large: %ld entries", nent);
    int pairbits = 1;
    while ((1L << pairbits) < npairs) ++pairbits;
    MM_REQUIRE(33 + pairbits <= 64, "adjoint table too large: %ld cell pairs", npairs);
    unsigned long long *kin = nullptr, *kout = nullptr;
    unsigned *head = nullptr, *pos = nullptr, *pairs = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0, scan_bytes = 0;
    int rc = MM_OK;
    auto cleanup = [&]() {
        void* bufs[] = {kin, kout, head, pos, pairs, tmp};
        for (void* b : bufs)
            if (b) cudaFree(b);
    };
    auto fail = [&](int r) {
        cleanup();
        free_table(h, tb);
        return r;
    };
    auto fail_cuda = [&](cudaError_t e) {
        mm::set_error("building the adjoint scatter table: %s", cudaGetErrorString(e));
        return fail(MM_ECUDA);
    };
    if ((rc = dev_alloc((void**)&kin, nent * 8, "scatter keys")) != MM_OK) return fail(rc);
    if ((rc = dev_alloc((void**)&kout, nent * 8, "scatter keys (sorted)")) != MM_OK) return fail(rc);
    if ((rc = dev_alloc((void**)&head, nent * 4, "scatter merge flags")) != MM_OK) return fail(rc);
    if ((rc = dev_alloc((void**)&pos, nent * 4, "scatter entry positions")) != MM_OK) return fail(rc);
    cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, kin, kout, (int64_t)nent, 0, 33 + pairbits, st);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, head, pos, (int64_t)nent, st);
    tmp_bytes = std::max(tmp_bytes, scan_bytes);
    if ((rc = dev_alloc(&tmp, tmp_bytes, "sort/scan temp")) != MM_OK) return fail(rc);
    const long gb = (nent + kThreads - 1) / kThreads;
    const float scale = (float)(1.0 / (4.0 * n * (double)n));
#define MM_K(MM)                                                                         \
    case MM:                                                                             \
        k_pair_keys<MM><<<gb, kThreads, 0, st>>>(kin, h->d_cos, h->d_sin, n, T, nent, e0); \
        break;
    switch (M) {
        MM_K(2) MM_K(3) MM_K(4) MM_K(5) MM_K(6)
        default: mm::set_error("unsupported m=%d", M); return fail(MM_EINVAL);
    }
#undef MM_K
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, kin, kout, (int64_t)nent, 0, 33 + pairbits, st);
    if (e == cudaSuccess) {
#define MM_H(MM) \
    case MM: k_pair_heads<MM><<<gb, kThreads, 0, st>>>(kout, head, nent); break;
        switch (M) { MM_H(2) MM_H(3) MM_H(4) MM_H(5) MM_H(6) }
#undef MM_H
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, head, pos, (int64_t)nent, st);
    unsigned last_pos = 0, last_head = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_pos, pos + nent - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&last_head, head + nent - 1, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(e);
    const long nnz = (long)last_pos + last_head;
    if ((rc = talloc(h, tb, &tb.ptr, npairs + 1, "scatter pair pointers")) != MM_OK) return fail(rc);
    if ((rc = talloc(h, tb, &tb.idx, std::max(nnz, 1L), "scatter sample index")) != MM_OK) return fail(rc);
    if ((rc = talloc(h, tb, &tb.w, std::max(nnz, 1L), "scatter weights")) != MM_OK) return fail(rc);
    if ((rc = dev_alloc((void**)&pairs, std::max(nnz, 1L) * 4, "scatter entry pairs")) != MM_OK) return fail(rc);
#define MM_P(MM)                                                                                                 \
    case MM:                                                                                                     \
        k_pair_payload<MM><<<gb, kThreads, 0, st>>>(kout, head, pos, tb.idx, tb.w, pairs, h->d_cos, h->d_sin, n, T, \
                                                    nent, e0, h->c0, h->c1, scale);                              \
        break;
    switch (M) { MM_P(2) MM_P(3) MM_P(4) MM_P(5) MM_P(6) }
#undef MM_P
    k_pair_ptr<<<(nnz + 1 + kThreads - 1) / kThreads, kThreads, 0, st>>>(pairs, tb.ptr, nnz, npairs);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(e);
    cleanup();
    kin = kout = nullptr;
    head = pos = pairs = nullptr;
    tmp = nullptr;
    // long lists -> pieces of kChunk entries (fixed split: deterministic)
    std::vector<unsigned> hp(npairs + 1);
    MM_CUDA(cudaMemcpy(hp.data(), tb.ptr, hp.size() * sizeof(unsigned), cudaMemcpyDeviceToHost));
    std::vector<uint2> tasks;
    std::vector<uint4> longp;
    for (long q = 0; q < npairs; ++q) {
        const unsigned a = hp[q], b = hp[q + 1];
        if (b - a <= kChunk) continue;
        const unsigned t0 = (unsigned)tasks.size();
        for (unsigned x = a; x < b; x += kChunk) tasks.push_back(make_uint2(x, std::min(b, x + kChunk)));
        longp.push_back(make_uint4((unsigned)q, t0, (unsigned)tasks.size(), 0u));
    }
    if (!longp.empty()) {
        if ((rc = talloc(h, tb, &tb.chunk_task, tasks.size(), "scatter pieces")) != MM_OK ||
            (rc = talloc(h, tb, &tb.chunk_pair, longp.size(), "scatter long pairs")) != MM_OK ||
            (rc = talloc(h, tb, &tb.chunk_part, tasks.size() * 2 * (size_t)h->zs, "scatter partial sums")) != MM_OK)
            return fail(rc);
        if (cudaMemcpy(tb.chunk_task, tasks.data(), tasks.size() * sizeof(uint2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(tb.chunk_pair, longp.data(), longp.size() * sizeof(uint4), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail_cuda(cudaGetLastError());
    }
    tb.nchunks = (long)tasks.size();
    tb.nlong = (long)longp.size();
    tb.nnz = nnz;
    return MM_OK;
}

// Splits the angles into table blocks and decides whether the tables stay
// resident: each block's build needs about kBuildBytesPerTap bytes per tap,
// the blocks' tables together about 7 bytes per tap plus one pointer array
// (4 bytes per cell pair) each.  The blocks are sized to a third of the free
// device memory (and to opts.max_table_angles); when all their tables would
// take more than half of it they are built at every RT call instead.
int build_csr(mm_tomo* h, cudaStream_t st) {
    if (h->csr_ready) return MM_OK;
    const int T = h->ntheta, L = 2 * h->m + 1;
    const long per_angle = (long)h->K * L * L;
    const long npairs = 2L * h->n * (h->n / 2 + 1);
    size_t freeb = 0, totalb = 0;
    MM_CUDA(cudaMemGetInfo(&freeb, &totalb));
    long tb = std::max(1L, std::min((long)T, ((1L << 32) - 1) / per_angle));
    tb = std::max(1L, std::min(tb, (long)(freeb / 3 / kBuildBytesPerTap) / per_angle));
    if (h->table_angles > 0) tb = std::min(tb, (long)h->table_angles);
    const long nblocks = (T + tb - 1) / tb;
    const double resident = 7.0 * per_angle * T + 4.0 * (npairs + 1) * nblocks;
    h->tables_resident = resident <= 0.5 * (double)freeb;
    h->tabs.assign(nblocks, ScatterTable());
    for (long b = 0; b < nblocks; ++b) {
        h->tabs[b].t0 = (int)(b * tb);
        h->tabs[b].t1 = (int)std::min((long)T, (b + 1) * tb);
    }
    if (h->tables_resident) {
        h->tm.begin(12, st);
        for (auto& t : h->tabs) {
            const int rc = build_table(h, t, st);
            if (rc != MM_OK) {
                for (auto& u : h->tabs) free_table(h, u);
                h->tabs.clear();
                return rc;
            }
        }
        h->tm.end(st, 4 * (int)h->tabs.size());
    }
    h->csr_ready = true;
    return MM_OK;
}

// The scatter of all angle blocks into A, in block order: the first block's
// sums are stored, every later block's are added.
int launch_scatter(mm_tomo* h, const float2* Q, float2* A, cudaStream_t st) {
    for (size_t b = 0; b < h->tabs.size(); ++b) {
        ScatterTable& t = h->tabs[b];
        if (!h->tables_resident) MM_TRY(build_table(h, t, st));
        const int rc = launch_table(h, t, Q, A, b > 0 ? 1 : 0, st);
        if (!h->tables_resident) {
            cudaStreamSynchronize(st);
            free_table(h, t);
        }
        MM_TRY(rc);
    }
    return MM_OK;
}

}  // namespace

namespace mmtomo {
int build_csr(mm_tomo* h, cudaStream_t st) { return ::build_csr(h, st); }
void free_tables(mm_tomo* h) {
    for (auto& t : h->tabs) ::free_table(h, t);
    h->tabs.clear();
    h->csr_ready = false;
}
int launch_scatter(mm_tomo* h, const float2* Q, float2* A, cudaStream_t st) { return ::launch_scatter(h, Q, A, st); }
}  // namespace mmtomo
