// sell.cuh — the SELL path of a FUSED pass: short rows in slices of 32 sorted by length
// inside windows (SELL-C-σ), warp rows as a stream of 32-entry chunks.
//
// Short rows (at most SEQ_MAX entries). The rows are cut into windows of SELL_WIN
// consecutive rows; inside a window they are ordered by decreasing length (a stable order:
// ties keep row order) and the ordered rows are cut into slices of 32. A slice stores the
// entries of its rows column-major (entry j of the slice's row at position `lane` sits at
// off + 32·j + lane), padded to its longest row, so lane `lane` of a warp walks its own row
// with loads that are coalesced across the warp, gathers the vector and sums in registers.
// Sorting keeps the padding — and the partly used sectors of the index/value loads — small
// where row lengths vary. One CTA takes a window (k_sell_win): its warps sum the window's
// slices, leave each sum in shared memory at the row's place in the window, and after one
// barrier the CTA's threads run the epilogue in row order (row inputs and outputs coalesced).
//
// Warp rows (longer than SEQ_MAX, at most TILE_NNZ). Each is stored as whole chunks of 32
// entries (the last one padded with column -1), the rows one after another in row order;
// lane `lane` of a chunk holds entry lane + 32·chunk of its row. The chunks are cut into
// blocks of SELL_SEG_CHUNKS; a warp takes the rows that start in one block — a segment, at
// most SELL_SEG_CHUNKS / 2 rows since each has at least two chunks — (k_sell_rows) and
// streams their chunks BH at a time, the next batch's index/value loads issued before this
// batch's sums, so neither row boundaries nor the index loads stall the gathers; at each
// row's end the warp folds its lanes' partials with the fixed shuffle tree and the lane
// holding that row's inputs runs its epilogue. On a large pass the two kernels write
// disjoint rows and run side by side on two streams; a small pass runs both in one launch
// (k_sell_both), whose fixed cost is one kernel.
//
// Both sums are the tile engine's: a short row from -0.0 in column order by one thread, a
// warp row as lane-strided partials (lane k: entries k, k + 32, … in order) and the same
// tree; so all engines give the same bits. The path is built only for matrices without rows
// longer than TILE_NNZ (those need the CTA-wide tree).
#pragma once

#include "tiles.cuh"

namespace sp {

constexpr int64_t SELL_MAX_SLOTS_PER_NNZ = 2;  // padding cap of a SELL copy (server footprints count it)
constexpr uint8_t SELL_HEAVY = 0xFF;           // length mark of a warp row
constexpr int SELL_WIN_SHIFT = 9;
// Rows per window: one CTA's work (the 40M LP's dual pass, ms FP64 / FP32: 256 rows 0.197 /
// 0.182, 512 0.188 / 0.182, 1,024 0.193 / 0.190).
constexpr int SELL_WIN = 1 << SELL_WIN_SHIFT;
constexpr int SELL_SPW = SELL_WIN / 32 / (NT / 32);  // slices per warp in a window
// Chunks per block: a warp takes the rows starting in one (the 40M LP's primal pass on this
// path, ms: blocks of 8 0.316, 16 0.279, 32 0.267, 48 0.268, 62 0.270).
constexpr int SELL_SEG_CHUNKS = 32;
static_assert(SELL_WIN % NT == 0 && SELL_SPW >= 1, "a window is a whole number of slices per warp");
static_assert(SELL_SEG_CHUNKS / 2 < 32, "a segment's row bounds sit in one lane each");

struct SellMat {
    int64_t nrows = 0, nwin = 0, nslices = 0, slots = 0;
    int64_t nheavy = 0, nseg = 0, chunks = 0;
    bool split = false;         // rows and windows as two launches on two streams (a large pass)
    int *ci = nullptr;          // [slots] slices
    double *v = nullptr;        // [slots]
    float *v32 = nullptr;       // [slots], mixed form
    int64_t *off = nullptr;     // [nslices] first slot of each slice
    int *slen = nullptr;        // [nslices] longest row of each slice
    uint8_t *len = nullptr;     // [nwin * SELL_WIN] row lengths in row order, SELL_HEAVY for warp rows
    uint8_t *lsort = nullptr;   // [nwin * SELL_WIN] short row lengths in slice order (warp rows 0)
    uint16_t *perm = nullptr;   // [nwin * SELL_WIN] row (within its window) at each slice position
    int *heavy = nullptr;       // [nheavy] the warp rows, in row order
    int64_t *choff = nullptr;   // [nheavy + 1] first chunk of each warp row
    int *segrow = nullptr;      // [nseg + 1] first warp row of each segment
    int *hci = nullptr;         // [chunks * 32] warp rows' columns, -1 past a row's end
    double *hv = nullptr;       // [chunks * 32]
    float *hv32 = nullptr;      // [chunks * 32], mixed form
    bool ok = false;
};

// Pointers of the SELL copy the kernels read.
struct SellArgs {
    const int *ci;
    const double *v;
    const float *v32;
    const int64_t *off;
    const int *slen;
    const uint8_t *len, *lsort;
    const uint16_t *perm;
    const int *heavy;
    const int64_t *choff;
    const int *segrow;
    const int *hci;
    const double *hv;
    const float *hv32;
    int64_t nrows, nwin, nheavy, nseg;
};

// Per row (the last window padded with empty rows): its length mark in row order, its
// warp-row flag, and its sort key — the window, then 32 minus its short length — so that a
// stable sort of the keys orders each window's rows by decreasing short length (warp rows
// and padding count as 0) and keeps row order among equal lengths.
__global__ void k_sell_keys(const int *__restrict__ rp, int64_t nrows, int64_t npad, uint8_t *__restrict__ len,
                            int *__restrict__ heavy_flag, uint32_t *__restrict__ key, uint16_t *__restrict__ loc) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < npad; r += (int64_t)gridDim.x * blockDim.x) {
        const int l = r < nrows ? rp[r + 1] - rp[r] : 0;
        const bool heavy = l > SEQ_MAX;
        len[r] = heavy ? SELL_HEAVY : (uint8_t)l;
        if (r < nrows) heavy_flag[r] = heavy ? 1 : 0;
        key[r] = ((uint32_t)(r >> SELL_WIN_SHIFT) << 6) | (uint32_t)(32 - (heavy ? 0 : l));
        loc[r] = (uint16_t)(r & (SELL_WIN - 1));
    }
}

// Per slice position of the sorted keys: the short length there; per slice its width (its
// first row is its longest) and slot count.
__global__ void k_sell_slices(const uint32_t *__restrict__ skey, int64_t npad, uint8_t *__restrict__ lsort,
                              int *__restrict__ slen, int64_t *__restrict__ slots) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < npad; k += (int64_t)gridDim.x * blockDim.x) {
        const int l = 32 - (int)(skey[k] & 63u);
        lsort[k] = (uint8_t)l;
        if ((k & 31) == 0) {
            slen[k >> 5] = l;
            slots[k >> 5] = 32ll * l;
        }
    }
}

// Per warp row: its chunk count (entry h of nheavy + 1; the last is 0, for the scan's total).
__global__ void k_sell_chunk_counts(const int *__restrict__ rp, const int *__restrict__ heavy, int64_t nheavy,
                                    int64_t *__restrict__ cnt) {
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h <= nheavy; h += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = 0;
        if (h < nheavy) {
            const int r = heavy[h];
            c = (rp[r + 1] - rp[r] + 31) / 32;
        }
        cnt[h] = c;
    }
}

// Per segment k (and the end, k = nseg): its first warp row, the first whose first chunk is
// at or past k·SELL_SEG_CHUNKS (a binary search over the chunk offsets).
__global__ void k_sell_segments(const int64_t *__restrict__ choff, int64_t nheavy, int64_t nseg,
                                int *__restrict__ segrow) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= nseg; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = k * SELL_SEG_CHUNKS;
        int64_t lo = 0, hi = nheavy;  // choff[nheavy] is the total: every block start is at most it
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (choff[mid] < c) lo = mid + 1;
            else hi = mid;
        }
        segrow[k] = (int)(k == nseg ? nheavy : lo);
    }
}

// One thread per slice position: copies its row's entries to their column-major slots.
__global__ void k_sell_fill(const int *__restrict__ rp, const int *__restrict__ ci, const double *__restrict__ v,
                            int64_t npad, const uint8_t *__restrict__ lsort, const uint16_t *__restrict__ perm,
                            const int64_t *__restrict__ off, int *__restrict__ sci, double *__restrict__ sv,
                            float *__restrict__ sv32) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < npad; k += (int64_t)gridDim.x * blockDim.x) {
        const int l = lsort[k];
        if (l == 0) continue;
        const int64_t r = ((k >> SELL_WIN_SHIFT) << SELL_WIN_SHIFT) + perm[k];
        const int a = rp[r];
        const int64_t o = off[k >> 5] + (k & 31);
        for (int j = 0; j < l; ++j) {
            const int64_t d = o + 32ll * j;
            sci[d] = ci[a + j];
            sv[d] = v[a + j];
            if (sv32) sv32[d] = (float)v[a + j];
        }
    }
}

// One warp per warp row: copies its entries to its chunks, padding the last with column -1.
__global__ void k_sell_chunk_fill(const int *__restrict__ rp, const int *__restrict__ ci, const double *__restrict__ v,
                                  const int *__restrict__ heavy, int64_t nheavy, const int64_t *__restrict__ choff,
                                  int *__restrict__ hci, double *__restrict__ hv, float *__restrict__ hv32) {
    const int lane = threadIdx.x & 31;
    for (int64_t h = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; h < nheavy;
         h += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int r = heavy[h];
        const int a = rp[r], l = rp[r + 1] - a;
        const int64_t base = choff[h] * 32;
        const int n = (int)(choff[h + 1] - choff[h]) * 32;
        for (int j = lane; j < n; j += 32) {
            const bool in = j < l;
            hci[base + j] = in ? ci[a + j] : -1;
            const double x = in ? v[a + j] : 0.0;
            hv[base + j] = x;
            if (hv32) hv32[base + j] = (float)x;
        }
    }
}

// The warp rows of segment `seg` of a FUSED pass (NP = 0, one gathered vector) on the SELL
// copy, by one warp: up to 2·BH chunks in flight per lane.
template <class Op, int BH>
__device__ __forceinline__ void sell_rows_body(Op &op, const SellArgs &S, int64_t seg) {
    using VT = typename Op::VT;
    using GT = typename Op::GT;
    using Pre = typename Op::Pre;
    static_assert(Op::G == 1 && Op::NP == 0, "the SELL path runs passes that gather one vector and reduce nothing");
    constexpr bool F32 = (Op::F32 & 1u) != 0;
    using AT = typename std::conditional<F32, float, double>::type;
    const int lane = threadIdx.x & 31;
    const GT *__restrict__ gv = op.gvec();
    double part[1] = {0.0};
    const int64_t h0 = S.segrow[seg];
    const int nr = S.segrow[seg + 1] - (int)h0;
    if (nr == 0) return;  // a block inside one long row
    // lane k < nr: row k of the segment and its inputs; lanes 0..nr: the chunk bounds
    int row = 0;
    int64_t bound = 0;
    Pre pre{};
    if (lane <= nr) bound = S.choff[h0 + lane];
    if (lane < nr) {
        row = S.heavy[h0 + lane];
        pre = op.pre(row);
    }
    const int64_t c0 = __shfl_sync(0xffffffffu, bound, 0), c1 = __shfl_sync(0xffffffffu, bound, nr);
    const VT *__restrict__ hv;
    if constexpr (sizeof(VT) == 4) hv = reinterpret_cast<const VT *>(S.hv32);
    else hv = reinterpret_cast<const VT *>(S.hv);
    int cur = 0;
    AT s = AT(-0.0);
    // row cur is complete: the tree, then its epilogue on the lane that holds it
    auto finish = [&]() {
        const AT tot = __shfl_sync(0xffffffffu, warp_sum_down(s), 0);
        if (lane == cur) {
            const double sum[1] = {double(tot)};
            op.row(row, sum, part, pre);
        }
    };
    const int *__restrict__ pc = S.hci + c0 * 32 + lane;
    const VT *__restrict__ pv = hv + c0 * 32 + lane;
    const int nch = (int)(c1 - c0);
    int nxt = (int)(__shfl_sync(0xffffffffu, bound, 1) - c0);  // first chunk of row cur + 1
    int c[BH];
    VT v[BH];
#pragma unroll
    for (int u = 0; u < BH; ++u) {
        c[u] = -1;
        if (u < nch) {
            c[u] = ld_stream(pc + 32 * u);
            v[u] = ld_stream(pv + 32 * u);
        }
    }
    for (int ch = 0; ch < nch; ch += BH) {
        GT g[BH];
#pragma unroll
        for (int u = 0; u < BH; ++u)
            if (c[u] >= 0) g[u] = __ldg(gv + c[u]);
        pc += 32 * BH;
        pv += 32 * BH;
        int cn[BH];
        VT vn[BH];
#pragma unroll
        for (int u = 0; u < BH; ++u) {
            cn[u] = -1;
            if (ch + BH + u < nch) {
                cn[u] = ld_stream(pc + 32 * u);
                vn[u] = ld_stream(pv + 32 * u);
            }
        }
#pragma unroll
        for (int u = 0; u < BH; ++u) {
            if (ch + u >= nch) break;
            if (ch + u == nxt) {  // a warp row spans at least two chunks
                finish();
                ++cur;
                nxt = (int)(__shfl_sync(0xffffffffu, bound, cur + 1) - c0);
                s = AT(-0.0);
            }
            if (c[u] >= 0) s += AT(op.mul(v[u], g[u]));
        }
#pragma unroll
        for (int u = 0; u < BH; ++u) {
            c[u] = cn[u];
            v[u] = vn[u];
        }
    }
    finish();
}

// The warp rows of a FUSED pass on the SELL copy: one segment per warp; MINB CTAs per SM.
template <class Op, int BH, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_sell_rows(Op op, SellArgs S) {
    if (!op.setup()) return;
    const int64_t seg = (int64_t)blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
    if (seg < S.nseg) sell_rows_body<Op, BH>(op, S, seg);
}

// The short rows of window `win` of a FUSED pass (NP = 0, one gathered vector) on the SELL
// copy, by one CTA: BS slice entries in flight per lane.
template <class Op, int BS>
__device__ __forceinline__ void sell_win_body(Op &op, const SellArgs &S, int64_t win) {
    using VT = typename Op::VT;
    using GT = typename Op::GT;
    using Pre = typename Op::Pre;
    static_assert(Op::G == 1 && Op::NP == 0, "the SELL path runs passes that gather one vector and reduce nothing");
    constexpr bool F32 = (Op::F32 & 1u) != 0;
    using AT = typename std::conditional<F32, float, double>::type;
    constexpr int W = NT / 32;  // warps per CTA
    __shared__ AT sums[SELL_WIN];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const GT *__restrict__ gv = op.gvec();
    double part[1] = {0.0};
    const VT *__restrict__ sv;
    if constexpr (sizeof(VT) == 4) sv = reinterpret_cast<const VT *>(S.v32);
    else sv = reinterpret_cast<const VT *>(S.v);
    // the window's slices, widest first, dealt to the warps back and forth so that each
    // warp's widths add up to about the same
#pragma unroll 1
    for (int q = 0; q < SELL_SPW; ++q) {
        const int ls = q * W + ((q & 1) ? W - 1 - warp : warp);
        const int64_t sl = win * (SELL_WIN / 32) + ls;
        const int64_t k = sl * 32 + lane;
        const int l = S.lsort[k];
        const int L = S.slen[sl];
        const int64_t off = S.off[sl] + lane;
        AT s = AT(-0.0);
        for (int j0 = 0; j0 < L; j0 += BS) {
            int c[BS];
            VT v[BS];
#pragma unroll
            for (int u = 0; u < BS; ++u) {
                if (j0 + u < l) {
                    c[u] = ld_stream(S.ci + off + 32ll * (j0 + u));
                    v[u] = ld_stream(sv + off + 32ll * (j0 + u));
                }
            }
#pragma unroll
            for (int u = 0; u < BS; ++u)
                if (j0 + u < l) s += AT(op.mul(v[u], __ldg(gv + c[u])));
        }
        sums[S.perm[k]] = s;
    }
    // the epilogue in row order, row inputs loaded before the barrier
    constexpr int RPT = SELL_WIN / NT;
    const int64_t rbase = win * SELL_WIN + threadIdx.x;
    Pre pre[RPT];
    bool live[RPT];
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
        const int64_t r = rbase + u * NT;
        live[u] = r < S.nrows && S.len[r] != SELL_HEAVY;
        if (live[u]) pre[u] = op.pre((int)r);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < RPT; ++u) {
        if (!live[u]) continue;
        const double sum[1] = {double(sums[threadIdx.x + u * NT])};
        op.row((int)(rbase + u * NT), sum, part, pre[u]);
    }
}

// The short rows of a FUSED pass on the SELL copy: one window per CTA; MINB CTAs per SM.
template <class Op, int BS, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_sell_win(Op op, SellArgs S) {
    if (!op.setup()) return;
    sell_win_body<Op, BS>(op, S, blockIdx.x);
}

// Both parts of a small FUSED pass in one launch: the first ceil(nseg / 8) CTAs take the
// segments, the rest the windows.
template <class Op, int BH, int BS, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_sell_both(Op op, SellArgs S) {
    if (!op.setup()) return;
    const int64_t hb = (S.nseg + NT / 32 - 1) / (NT / 32);
    if ((int64_t)blockIdx.x < hb) {
        const int64_t seg = (int64_t)blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
        if (seg < S.nseg) sell_rows_body<Op, BH>(op, S, seg);
    } else {
        sell_win_body<Op, BS>(op, S, blockIdx.x - hb);
    }
}

}  // namespace sp

namespace sp {

// ---- check passes on the SELL copy -------------------------------------------------
//
// A pass with G product slots and NP partial sums across rows (the check iteration's dual
// pass) runs on the SELL copy in two launches. k_sell_chk sums every row's G slots exactly
// as the tile engine does (the same order per slot, the same tree for a warp row) and runs
// its epilogue with partial sums that start at zero, storing each row's NP contributions
// in `contrib` ([NP][nrows]). k_sell_refold then adds them up per tile in the tile
// engine's order — each thread its short rows, lane 0 of warp w the warp rows w, w + 8, …,
// then the block tree — and stores the tile's partials. A partial sum never becomes -0.0,
// so adding a contribution that started from +0.0 gives the bits the tile engine's
// in-place accumulation gives.

template <int G, unsigned F32>
struct SlotSums {
    float f[G];
    double d[G];
    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int q = 0; q < G; ++q) { f[q] = -0.0f; d[q] = -0.0; }
    }
    template <class ST>
    __device__ __forceinline__ void add(const ST (&p)[G]) {
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if ((F32 >> q) & 1u) f[q] += float(p[q]);
            else d[q] += double(p[q]);
        }
    }
    __device__ __forceinline__ double get(int q) const { return ((F32 >> q) & 1u) ? double(f[q]) : d[q]; }
};

// One row's epilogue with its partials from zero, stored as its contributions.
template <class Op>
__device__ __forceinline__ void row_contrib(const Op &op, int r, const double (&sum)[Op::G],
                                            const typename Op::Pre &pre, double *contrib, int64_t nrows) {
    double part[Op::NP];
#pragma unroll
    for (int q = 0; q < Op::NP; ++q) part[q] = 0.0;
    op.row(r, sum, part, pre);
#pragma unroll
    for (int q = 0; q < Op::NP; ++q) contrib[q * nrows + r] = part[q];
}

// Segments (warp rows) first, one per warp, BH chunks per batch; then the windows.
template <class Op, int BH, int BS>
__global__ void __launch_bounds__(NT) k_sell_chk(Op op, SellArgs S, double *contrib) {
    using VT = typename Op::VT;
    using ST = typename Op::ST;
    using Pre = typename Op::Pre;
    constexpr int G = Op::G;
    constexpr unsigned F32 = Op::F32;
    constexpr int W = NT / 32;
    __shared__ double sums[G * SELL_WIN];
    if (!op.setup()) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t hb = (S.nseg + W - 1) / W;
    const VT *__restrict__ hv;
    const VT *__restrict__ sv;
    if constexpr (sizeof(VT) == 4) {
        hv = reinterpret_cast<const VT *>(S.hv32);
        sv = reinterpret_cast<const VT *>(S.v32);
    } else {
        hv = reinterpret_cast<const VT *>(S.hv);
        sv = reinterpret_cast<const VT *>(S.v);
    }
    if ((int64_t)blockIdx.x < hb) {
        const int64_t seg = (int64_t)blockIdx.x * W + warp;
        if (seg >= S.nseg) return;
        const int64_t h0 = S.segrow[seg];
        const int nr = S.segrow[seg + 1] - (int)h0;
        if (nr == 0) return;
        int row = 0;
        int64_t bound = 0;
        Pre pre{};
        if (lane <= nr) bound = S.choff[h0 + lane];
        if (lane < nr) {
            row = S.heavy[h0 + lane];
            pre = op.pre(row);
        }
        const int64_t c0 = __shfl_sync(0xffffffffu, bound, 0), c1 = __shfl_sync(0xffffffffu, bound, nr);
        const int nch = (int)(c1 - c0);
        int cur = 0, nxt = (int)(__shfl_sync(0xffffffffu, bound, 1) - c0);
        SlotSums<G, F32> acc;
        acc.clear();
        auto finish = [&]() {
            double tot[G];
#pragma unroll
            for (int q = 0; q < G; ++q) {
                if ((F32 >> q) & 1u) tot[q] = double(__shfl_sync(0xffffffffu, warp_sum_down(acc.f[q]), 0));
                else tot[q] = __shfl_sync(0xffffffffu, warp_sum_down(acc.d[q]), 0);
            }
            if (lane == cur) row_contrib(op, row, tot, pre, contrib, S.nrows);
        };
        for (int ch = 0; ch < nch; ch += BH) {
            int c[BH];
            VT v[BH];
            ST p[BH][G];
#pragma unroll
            for (int u = 0; u < BH; ++u) {
                c[u] = -1;
                if (ch + u < nch) {
                    c[u] = ld_stream(S.hci + (c0 + ch + u) * 32 + lane);
                    v[u] = ld_stream(hv + (c0 + ch + u) * 32 + lane);
                }
            }
#pragma unroll
            for (int u = 0; u < BH; ++u)
                if (c[u] >= 0) op.prod(c[u], v[u], p[u]);
#pragma unroll
            for (int u = 0; u < BH; ++u) {
                if (ch + u >= nch) break;
                if (ch + u == nxt) {  // a warp row spans at least two chunks
                    finish();
                    ++cur;
                    nxt = (int)(__shfl_sync(0xffffffffu, bound, cur + 1) - c0);
                    acc.clear();
                }
                if (c[u] >= 0) acc.add(p[u]);
            }
        }
        finish();
        return;
    }
    const int64_t win = blockIdx.x - hb;
#pragma unroll 1
    for (int qs = 0; qs < SELL_SPW; ++qs) {
        const int ls = qs * W + ((qs & 1) ? W - 1 - warp : warp);
        const int64_t sl = win * (SELL_WIN / 32) + ls;
        const int64_t k = sl * 32 + lane;
        const int l = S.lsort[k];
        const int L = S.slen[sl];
        const int64_t off = S.off[sl] + lane;
        SlotSums<G, F32> acc;
        acc.clear();
        for (int j0 = 0; j0 < L; j0 += BS) {
            int c[BS];
            VT v[BS];
            ST p[BS][G];
#pragma unroll
            for (int u = 0; u < BS; ++u) {
                if (j0 + u < l) {
                    c[u] = ld_stream(S.ci + off + 32ll * (j0 + u));
                    v[u] = ld_stream(sv + off + 32ll * (j0 + u));
                }
            }
#pragma unroll
            for (int u = 0; u < BS; ++u)
                if (j0 + u < l) op.prod(c[u], v[u], p[u]);
#pragma unroll
            for (int u = 0; u < BS; ++u)
                if (j0 + u < l) acc.add(p[u]);
        }
        const int at = S.perm[k];
#pragma unroll
        for (int q = 0; q < G; ++q) sums[q * SELL_WIN + at] = acc.get(q);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < SELL_WIN; t += NT) {
        const int64_t r = win * SELL_WIN + t;
        if (r >= S.nrows) break;
        if (S.len[r] == SELL_HEAVY) continue;
        double tot[G];
#pragma unroll
        for (int q = 0; q < G; ++q) tot[q] = sums[q * SELL_WIN + t];
        row_contrib(op, (int)r, tot, op.pre((int)r), contrib, S.nrows);
    }
}

// The tile partials of a k_sell_chk pass from its contributions, one CTA per tile (the
// matrix has no tile of a single row longer than TILE_NNZ: it has a SELL copy).
template <class Op>
__global__ void __launch_bounds__(NT) k_sell_refold(Op op, const uint8_t *__restrict__ len,
                                                    const double *__restrict__ contrib, int64_t nrows) {
    constexpr int NP = Op::NP;
    __shared__ double sh[NP * (NT / 32)];
    if (!op.setup()) return;
    const int tile = blockIdx.x, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Tile t = op.tiles[tile];
    const int r0 = t.x, nr = t.y - t.x;
    double part[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) part[q] = 0.0;
    auto add = [&](int64_t r) {
#pragma unroll
        for (int q = 0; q < NP; ++q) part[q] += contrib[q * nrows + r];
    };
    // short rows: thread u takes rows u, u + NT, …
    for (int u = tid; u < nr; u += NT)
        if (len[r0 + u] != SELL_HEAVY) add(r0 + u);
    // warp rows: warp w the rows w, w + 8, … in increasing order, on lane 0
    for (int base = warp; base < nr; base += 32 * (NT / 32)) {
        const int i = base + lane * (NT / 32);
        const bool heavy = i < nr && len[r0 + i] == SELL_HEAVY;
        for (unsigned mask = __ballot_sync(0xffffffffu, heavy); mask; mask &= mask - 1)
            if (lane == 0) add(r0 + base + (__ffs(mask) - 1) * (NT / 32));
    }
    __syncthreads();
    block_sum<NP>(part, sh);
    if (tid == 0) op.store(tile, part);
}

}  // namespace sp
