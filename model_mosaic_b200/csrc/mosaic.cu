// Mosaic tile extraction (step4_extract.py) and tent-weighted stitching
// (step6_stitch.py) for sm_100a.
//
// A placement p is one detector footprint in the big projection (NZ, N):
// rows [r_lo, r_lo + h), direct columns [cd, cd + w), mirror columns
// [cm, cm + w) (step4_extract.py:52-118).  Tiles are float32 frames (h, w).
//
// Extract (step4_extract.py:176-192): direct[p][t][i][j] = proj[t][r_lo+i][cd+j]
// and mirror[p][t][i][j] = proj[t][r_lo+i][cm+w-1-j] (the h-flipped mirror
// crop).  One block per tile row, looping over the angles: coalesced row
// reads and writes, no shared memory.
//
// Stitch (step6_stitch.py:206-262): the reference adds every placement's
// tent-weighted tile into a zeroed buffer and a weight plane, then divides.
// Here each output pixel pulls its covering placements instead, in the
// reference's order (placement order, direct before mirror), with the same
// float32 roundings (products and sums not contracted into FMAs, IEEE
// reciprocal), so the result is bit-identical while the output is written
// once and every tile pixel read once.  Coverage is constant on the cells
// of the grid cut by all footprint edges: a row-cell and a column-cell table
// give each pixel its cell, and a CSR list gives the cell's (placement,
// mirror) entries.  A thread owns one pixel for all angles of the call, so
// the entry setup and the reciprocal are paid once per pixel.
#include "mm_common.cuh"

#include <algorithm>
#include <vector>

using mm::dev_alloc;

namespace {

constexpr int kMaxPlace = 240;  // 2 * 240 tile pointers fit the 4 KB parameter space
constexpr int kThreads = 256;
constexpr int kAngles = 8;  // angles per batch of loads in the extract and stitch loops

struct Rect {
    int r_lo, h, cd, cm, w;
};

// Tile frame pointers of one call, passed by value: [0, np) direct, then mirror.
struct TilePtrs {
    float* p[2 * kMaxPlace];
};

}  // namespace

struct mm_mosaic {
    int nz = 0, n = 0, np = 0, cap = 0;
    int ncells_r = 0, ncells_c = 0, max_cover = 0;
    long ext_rows = 0;
    Rect* rect = nullptr;       // np
    int* rowcell = nullptr;     // nz
    int* colcell = nullptr;     // n
    int* cellptr = nullptr;     // ncells + 1
    int* cellent = nullptr;     // entries: p << 1 | mirror
    int2* extrow = nullptr;     // ext_rows: (p << 1 | mirror, i)
    std::vector<Rect> hrect;
    size_t ws_bytes = 0;
};

namespace {

// Tent weight of step6_stitch.py:70-81 at offset i of an extent h, cap c:
// min(min(i + 1/2, h - (i + 1/2)), c), every step exact in float32 for the
// integer sizes a detector has.
__device__ __forceinline__ float tent(int i, int h, float cap) {
    const float y = (float)i + 0.5f;
    return fminf(fminf(y, (float)h - y), cap);
}

__global__ void __launch_bounds__(kThreads) k_extract(const float* __restrict__ proj, TilePtrs dst,
                                                      const Rect* __restrict__ rect,
                                                      const int2* __restrict__ extrow, int np, int nz, int n,
                                                      int nth) {
    const int2 er = __ldg(extrow + blockIdx.x);
    const int p = er.x >> 1, mir = er.x & 1, i = er.y;
    const Rect rc = rect[p];
    const long fr = (long)rc.h * rc.w, plane = (long)nz * n;
    float* d = dst.p[mir * np + p] + (long)i * rc.w;
    const float* s = proj + (long)(rc.r_lo + i) * n;
    for (int j = threadIdx.x; j < rc.w; j += kThreads) {
        const float* sj = s + (mir ? rc.cm + rc.w - 1 - j : rc.cd + j);
        float* dj = d + j;
        int t = 0;
        for (; t + kAngles <= nth; t += kAngles) {  // kAngles independent loads in flight
            float v[kAngles];
#pragma unroll
            for (int u = 0; u < kAngles; ++u) v[u] = __ldg(sj + (t + u) * plane);
#pragma unroll
            for (int u = 0; u < kAngles; ++u) __stcs(dj + (t + u) * fr, v[u]);
        }
        for (; t < nth; ++t) __stcs(dj + t * fr, __ldg(sj + t * plane));
    }
}

// MAXE: bound on the entries of any cell (registers hold one pointer and
// one weight per entry); U: angles whose loads are issued together.
template <int MAXE, int U>
__global__ void __launch_bounds__(kThreads) k_stitch(TilePtrs src, float* __restrict__ out,
                                                     const Rect* __restrict__ rect,
                                                     const int* __restrict__ rowcell,
                                                     const int* __restrict__ colcell,
                                                     const int* __restrict__ cellptr,
                                                     const int* __restrict__ cellent, int np, int nz, int n,
                                                     int ncc, int nth, int ncb, float cap) {
    const int r = blockIdx.x / ncb;
    const int c = (blockIdx.x % ncb) * kThreads + threadIdx.x;
    if (c >= n) return;
    const long plane = (long)nz * n;
    float* o = out + (long)r * n + c;
    const int cell = __ldg(rowcell + r) * ncc + __ldg(colcell + c);
    const int e0 = __ldg(cellptr + cell), ne = __ldg(cellptr + cell + 1) - e0;
    const float* ptr[MAXE];
    int fs[MAXE];  // frame size h * w (a detector frame has far fewer than 2^31 pixels)
    float wt[MAXE];
    float wsum = 0.f;
#pragma unroll
    for (int k = 0; k < MAXE; ++k) {
        ptr[k] = nullptr;
        fs[k] = 0;
        wt[k] = 0.f;
        if (k < ne) {
            const int ent = __ldg(cellent + e0 + k);
            const int p = ent >> 1, mir = ent & 1;
            const Rect rc = rect[p];
            const int i = r - rc.r_lo, j = c - (mir ? rc.cm : rc.cd);
            wt[k] = __fmul_rn(tent(i, rc.h, cap), tent(j, rc.w, cap));
            wsum = __fadd_rn(wsum, wt[k]);
            ptr[k] = src.p[mir * np + p] + (long)i * rc.w + (mir ? rc.w - 1 - j : j);
            fs[k] = rc.h * rc.w;
        }
    }
    if (!(wsum > 0.f)) {  // no placement covers the pixel: air transmission
        for (int t = 0; t < nth; ++t) o[t * plane] = 1.0f;
        return;
    }
    const float inv = __fdiv_rn(1.0f, wsum);
    int t = 0;
    for (; t + U <= nth; t += U) {
        float v[U][MAXE];
#pragma unroll
        for (int k = 0; k < MAXE; ++k)
            if (k < ne) {
#pragma unroll
                for (int u = 0; u < U; ++u) v[u][k] = __ldg(ptr[k] + u * fs[k]);
                ptr[k] += U * fs[k];
            }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < MAXE; ++k)
                if (k < ne) acc = __fadd_rn(acc, __fmul_rn(v[u][k], wt[k]));
            __stcs(o + (t + u) * plane, __fmul_rn(acc, inv));
        }
    }
    for (; t < nth; ++t) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < MAXE; ++k)
            if (k < ne) {
                acc = __fadd_rn(acc, __fmul_rn(__ldg(ptr[k]), wt[k]));
                ptr[k] += fs[k];
            }
        __stcs(o + t * plane, __fmul_rn(acc, inv));
    }
}

int build_tables(mm_mosaic* h) {
    const int np = h->np;
    std::vector<int> rb = {0, h->nz}, cb = {0, h->n};
    for (const Rect& r : h->hrect) {
        rb.push_back(r.r_lo);
        rb.push_back(r.r_lo + r.h);
        cb.push_back(r.cd);
        cb.push_back(r.cd + r.w);
        cb.push_back(r.cm);
        cb.push_back(r.cm + r.w);
    }
    std::sort(rb.begin(), rb.end());
    rb.erase(std::unique(rb.begin(), rb.end()), rb.end());
    std::sort(cb.begin(), cb.end());
    cb.erase(std::unique(cb.begin(), cb.end()), cb.end());
    const int nrc = (int)rb.size() - 1, ncc = (int)cb.size() - 1;
    std::vector<int> rowcell(h->nz), colcell(h->n);
    for (int k = 0; k < nrc; ++k)
        for (int r = rb[k]; r < rb[k + 1]; ++r) rowcell[r] = k;
    for (int k = 0; k < ncc; ++k)
        for (int c = cb[k]; c < cb[k + 1]; ++c) colcell[c] = k;
    std::vector<int> ptr(1, 0), ent;
    int maxc = 0;
    for (int a = 0; a < nrc; ++a)
        for (int b = 0; b < ncc; ++b) {
            const int r = rb[a], c = cb[b];
            int cnt = 0;
            for (int p = 0; p < np; ++p) {
                const Rect& q = h->hrect[p];
                if (r < q.r_lo || r >= q.r_lo + q.h) continue;
                if (c >= q.cd && c < q.cd + q.w) { ent.push_back(p << 1); ++cnt; }
                if (c >= q.cm && c < q.cm + q.w) { ent.push_back(p << 1 | 1); ++cnt; }
            }
            maxc = std::max(maxc, cnt);
            ptr.push_back((int)ent.size());
        }
    if (ent.empty()) ent.push_back(0);
    std::vector<int2> extrow;
    for (int p = 0; p < np; ++p)
        for (int mir = 0; mir < 2; ++mir)
            for (int i = 0; i < h->hrect[p].h; ++i) extrow.push_back(make_int2(p << 1 | mir, i));
    h->ncells_r = nrc;
    h->ncells_c = ncc;
    h->max_cover = maxc;
    h->ext_rows = (long)extrow.size();
    auto up = [&](void** d, const void* s, size_t bytes, const char* what) -> int {
        MM_TRY(dev_alloc(d, bytes, what));
        MM_CUDA(cudaMemcpy(*d, s, bytes, cudaMemcpyHostToDevice));
        h->ws_bytes += bytes;
        return MM_OK;
    };
    MM_TRY(up((void**)&h->rect, h->hrect.data(), h->hrect.size() * sizeof(Rect), "mosaic placements"));
    MM_TRY(up((void**)&h->rowcell, rowcell.data(), rowcell.size() * sizeof(int), "mosaic row cells"));
    MM_TRY(up((void**)&h->colcell, colcell.data(), colcell.size() * sizeof(int), "mosaic column cells"));
    MM_TRY(up((void**)&h->cellptr, ptr.data(), ptr.size() * sizeof(int), "mosaic cell lists"));
    MM_TRY(up((void**)&h->cellent, ent.data(), ent.size() * sizeof(int), "mosaic cell entries"));
    MM_TRY(up((void**)&h->extrow, extrow.data(), extrow.size() * sizeof(int2), "mosaic tile rows"));
    return MM_OK;
}

void destroy(mm_mosaic* h) {
    void* bufs[] = {h->rect, h->rowcell, h->colcell, h->cellptr, h->cellent, h->extrow};
    for (void* b : bufs)
        if (b) cudaFree(b);
    delete h;
}

int fill_ptrs(const mm_mosaic* h, float* const* dir, float* const* mir, TilePtrs& tp, const char* what) {
    for (int p = 0; p < h->np; ++p) {
        MM_REQUIRE(dir[p] != nullptr && mir[p] != nullptr, "%s: tile pointer %d is NULL", what, p);
        MM_REQUIRE(((uintptr_t)dir[p] % 4) == 0 && ((uintptr_t)mir[p] % 4) == 0, "%s: tile %d misaligned", what,
                   p);
        tp.p[p] = dir[p];
        tp.p[h->np + p] = mir[p];
    }
    return MM_OK;
}

}  // namespace

extern "C" int mm_mosaic_create(int nz, int n, int n_place, const int* rects, int overlap, mm_mosaic** out) {
    MM_REQUIRE(out != nullptr, "mm_mosaic_create: out is NULL");
    *out = nullptr;
    MM_REQUIRE(rects != nullptr, "mm_mosaic_create: rects is NULL");
    MM_REQUIRE(nz >= 1 && n >= 1 && (long)nz * n <= (1L << 40), "mm_mosaic_create: projection (%d, %d) out of range",
               nz, n);
    MM_REQUIRE(n_place >= 1 && n_place <= kMaxPlace, "mm_mosaic_create: %d placements (1..%d supported)", n_place,
               kMaxPlace);
    mm_mosaic* h = new mm_mosaic();
    h->nz = nz;
    h->n = n;
    h->np = n_place;
    h->cap = overlap;
    for (int p = 0; p < n_place; ++p) {
        const int* q = rects + 8 * p;  // r_lo_dir, r_hi_dir, c_lo_dir, c_hi_dir, r_lo_mir, r_hi_mir, c_lo_mir, c_hi_mir
        const bool ok = q[0] >= 0 && q[1] <= nz && q[1] > q[0] && q[2] >= 0 && q[3] <= n && q[3] > q[2] &&
                        q[4] == q[0] && q[5] == q[1] && q[6] >= 0 && q[7] <= n && q[7] - q[6] == q[3] - q[2];
        if (!ok) {
            mm::set_error("mm_mosaic_create: placement %d rows [%d, %d) cols [%d, %d) mirror rows [%d, %d) cols "
                          "[%d, %d) is empty, outside (%d, %d) or mismatched",
                          p, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], nz, n);
            delete h;
            return MM_EINVAL;
        }
        h->hrect.push_back(Rect{q[0], q[1] - q[0], q[2], q[6], q[3] - q[2]});
    }
    const int rc = build_tables(h);
    if (rc != MM_OK) {
        destroy(h);
        return rc;
    }
    if (h->max_cover > 32) {
        mm::set_error("mm_mosaic_create: %d footprints overlap one pixel (at most 32 supported)", h->max_cover);
        destroy(h);
        return MM_EINVAL;
    }
    *out = h;
    return MM_OK;
}

extern "C" int mm_mosaic_destroy(mm_mosaic* h) {
    if (!h) return MM_OK;
    cudaDeviceSynchronize();
    destroy(h);
    return MM_OK;
}

extern "C" int mm_mosaic_extract(mm_mosaic* h, const float* proj, int nth, float* const* dir, float* const* mir,
                                 void* stream) {
    MM_REQUIRE(h != nullptr, "mm_mosaic_extract: NULL handle");
    MM_REQUIRE(nth >= 0, "mm_mosaic_extract: nth=%d negative", nth);
    if (nth == 0) return MM_OK;
    MM_REQUIRE(proj != nullptr && dir != nullptr && mir != nullptr, "mm_mosaic_extract: NULL array");
    MM_REQUIRE(((uintptr_t)proj % 4) == 0, "mm_mosaic_extract: misaligned projection");
    TilePtrs tp;
    MM_TRY(fill_ptrs(h, dir, mir, tp, "mm_mosaic_extract"));
    k_extract<<<(unsigned)h->ext_rows, kThreads, 0, (cudaStream_t)stream>>>(proj, tp, h->rect, h->extrow, h->np,
                                                                            h->nz, h->n, nth);
    MM_LAUNCHED();
    return MM_OK;
}

extern "C" int mm_mosaic_stitch(mm_mosaic* h, float* const* dir, float* const* mir, int nth, float* out,
                                void* stream) {
    MM_REQUIRE(h != nullptr, "mm_mosaic_stitch: NULL handle");
    MM_REQUIRE(nth >= 0, "mm_mosaic_stitch: nth=%d negative", nth);
    if (nth == 0) return MM_OK;
    MM_REQUIRE(out != nullptr && dir != nullptr && mir != nullptr, "mm_mosaic_stitch: NULL array");
    MM_REQUIRE(((uintptr_t)out % 4) == 0, "mm_mosaic_stitch: misaligned output");
    TilePtrs tp;
    MM_TRY(fill_ptrs(h, dir, mir, tp, "mm_mosaic_stitch"));
    const int ncb = (h->n + kThreads - 1) / kThreads;
    const long blocks = (long)h->nz * ncb;
    MM_REQUIRE(blocks < (1L << 31), "mm_mosaic_stitch: projection too large for one launch");
    const cudaStream_t st = (cudaStream_t)stream;
#define MM_S(E, U)                                                                                              \
    k_stitch<E, U><<<(unsigned)blocks, kThreads, 0, st>>>(tp, out, h->rect, h->rowcell, h->colcell, h->cellptr, \
                                                       h->cellent, h->np, h->nz, h->n, h->ncells_c, nth, ncb,  \
                                                       (float)h->cap)
    if (h->max_cover <= 4)
        MM_S(4, kAngles);
    else if (h->max_cover <= 8)
        MM_S(8, kAngles / 2);
    else
        MM_S(32, 1);
#undef MM_S
    MM_LAUNCHED();
    return MM_OK;
}

extern "C" int mm_mosaic_info(const mm_mosaic* h, int* cells_r, int* cells_c, int* max_cover) {
    MM_REQUIRE(h != nullptr, "mm_mosaic_info: NULL handle");
    if (cells_r) *cells_r = h->ncells_r;
    if (cells_c) *cells_c = h->ncells_c;
    if (max_cover) *max_cover = h->max_cover;
    return MM_OK;
}

extern "C" size_t mm_mosaic_workspace_bytes(const mm_mosaic* h) { return h ? h->ws_bytes : 0; }
