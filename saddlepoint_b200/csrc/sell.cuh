// sell.cuh — the SELL-32 path of a FUSED pass over a matrix whose rows are short.
//
// The rows are cut into slices of 32 consecutive rows; a slice stores the entries of its
// rows column-major (entry j of the slice's row `lane` at off + 32·j + lane), padded to its
// longest row, so lane `lane` of a warp walks its own row with loads that are coalesced
// across the warp, gathers the vector and sums in registers: no shared memory, no
// barrier. Rows longer than SEQ_MAX are left out of the slices (length 0) and summed by
// one warp each straight from the CSR arrays. Both sums are the tile engine's: a short
// row from -0.0 in column order by one thread, a long row as lane-strided partials and
// the fixed shuffle tree; so all engines give the same bits. The path is built only for
// matrices without rows longer than TILE_NNZ (those need the CTA-wide tree).
#pragma once

#include "tiles.cuh"

namespace sp {

constexpr int64_t SELL_MAX_SLOTS_PER_NNZ = 2;  // padding cap of a SELL copy (server footprints count it)
constexpr uint8_t SELL_HEAVY = 0xFF;  // length mark of a row summed by a warp

struct SellMat {
    int64_t nrows = 0, nslices = 0, nheavy = 0, slots = 0;
    int *ci = nullptr;       // [slots]
    double *v = nullptr;     // [slots]
    float *v32 = nullptr;    // [slots], mixed form
    int64_t *off = nullptr;  // [nslices] first slot of each slice
    int *slen = nullptr;     // [nslices] longest short row of each slice
    uint8_t *len = nullptr;  // [nslices * 32] row lengths, SELL_HEAVY for warp rows
    int *heavy = nullptr;    // [nheavy] the warp rows
    bool ok = false;
};

// Pointers of the SELL copy the kernel reads.
struct SellArgs {
    const int *ci;
    const double *v;
    const float *v32;
    const int64_t *off;
    const int *slen;
    const uint8_t *len;
    const int *heavy;
    int64_t nrows, nslices, nheavy;
};

// One warp per slice: row lengths, warp rows flagged, the slice's longest short row and
// its slot count (32 per entry of that row).
__global__ void k_sell_meta(const int *__restrict__ rp, int64_t nrows, int64_t nslices, uint8_t *__restrict__ len,
                            int *__restrict__ slen, int64_t *__restrict__ slots, int *__restrict__ heavy_flag) {
    const int lane = threadIdx.x & 31;
    for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < nslices;
         s += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t r = s * 32 + lane;
        const int l = r < nrows ? rp[r + 1] - rp[r] : 0;
        const bool heavy = l > SEQ_MAX;
        const int ls = heavy ? 0 : l;
        len[r] = heavy ? SELL_HEAVY : (uint8_t)ls;
        if (r < nrows) heavy_flag[r] = heavy ? 1 : 0;
        const int mx = __reduce_max_sync(0xffffffffu, ls);
        if (lane == 0) {
            slen[s] = mx;
            slots[s] = 32ll * mx;
        }
    }
}

// One warp per slice: copies each short row's entries to its column-major slots.
__global__ void k_sell_fill(const int *__restrict__ rp, const int *__restrict__ ci, const double *__restrict__ v,
                            int64_t nrows, int64_t nslices, const uint8_t *__restrict__ len,
                            const int64_t *__restrict__ off, int *__restrict__ sci, double *__restrict__ sv,
                            float *__restrict__ sv32) {
    const int lane = threadIdx.x & 31;
    for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < nslices;
         s += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t r = s * 32 + lane;
        const int l = len[r];
        if (r >= nrows || l == SELL_HEAVY) continue;
        const int a = rp[r];
        for (int j = 0; j < l; ++j) {
            const int64_t d = off[s] + 32ll * j + lane;
            sci[d] = ci[a + j];
            sv[d] = v[a + j];
            if (sv32) sv32[d] = (float)v[a + j];
        }
    }
}

// A FUSED pass (NP = 0, one gathered vector) on the SELL copy: warps take the warp rows
// first, then the slices, one item each. B loads in flight per lane; MINB CTAs per SM.
template <class Op, int B, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_sell(Op op, SellArgs S) {
    using VT = typename Op::VT;
    using GT = typename Op::GT;
    using ST = typename Op::ST;
    using Pre = typename Op::Pre;
    static_assert(Op::G == 1 && Op::NP == 0, "the SELL path runs passes that gather one vector and reduce nothing");
    constexpr bool F32 = (Op::F32 & 1u) != 0;
    using AT = typename std::conditional<F32, float, double>::type;
    if (!op.setup()) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t item = (int64_t)blockIdx.x * (NT / 32) + warp;
    const GT *__restrict__ gv = op.gvec();
    double part[1] = {0.0};
    if (item < S.nheavy) {
        // a warp row straight from CSR: lane-strided partials in order, then the tree
        const int r = S.heavy[item];
        const int a = op.rp[r], b = op.rp[r + 1];
        AT s = AT(-0.0);
        for (int base = a + lane; base < b; base += 32 * B) {
            int c[B];
            VT v[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int e = base + 32 * u;
                if (e < b) {
                    c[u] = ld_stream(op.ci + e);
                    v[u] = ld_stream(op.vals + e);
                }
            }
#pragma unroll
            for (int u = 0; u < B; ++u)
                if (base + 32 * u < b) s += AT(op.mul(v[u], __ldg(gv + c[u])));
        }
        const double sum[1] = {double(warp_sum_down(s))};
        if (lane == 0) op.row(r, sum, part, op.pre(r));
        return;
    }
    const int64_t sl = item - S.nheavy;
    if (sl >= S.nslices) return;
    const int64_t r = sl * 32 + lane;
    const int lraw = S.len[r];
    const bool live = r < S.nrows && lraw != SELL_HEAVY;
    const int l = live ? lraw : 0;
    Pre pre{};
    if (live) pre = op.pre((int)r);
    const int L = S.slen[sl];
    const int64_t off = S.off[sl] + lane;
    const VT *__restrict__ sv;
    if constexpr (sizeof(VT) == 4) sv = reinterpret_cast<const VT *>(S.v32);
    else sv = reinterpret_cast<const VT *>(S.v);
    AT s = AT(-0.0);
    for (int j0 = 0; j0 < L; j0 += B) {
        int c[B];
        VT v[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
            if (j0 + u < l) {
                c[u] = ld_stream(S.ci + off + 32ll * (j0 + u));
                v[u] = ld_stream(sv + off + 32ll * (j0 + u));
            }
        }
#pragma unroll
        for (int u = 0; u < B; ++u)
            if (j0 + u < l) s += AT(op.mul(v[u], __ldg(gv + c[u])));
    }
    if (live) {
        const double sum[1] = {double(s)};
        op.row((int)r, sum, part, pre);
    }
}

}  // namespace sp
