// tiles.cuh — the row-tile CSR SpMV that every matrix pass of the PDHG is built on.
//
// A matrix is cut once, at load time, into tiles of consecutive rows holding at
// most TILE_NNZ nonzeros and TILE_ROWS rows; a row longer than TILE_NNZ gets a
// tile of its own. One CTA of NT threads processes one tile:
//   1. load: every load of the tile is issued before any of them is used — the
//      tile's row pointers, the inputs of the epilogue of this thread's first row
//      (Op::pre), and the TILE_NNZ / NT (column, value) pairs of this thread — so a
//      tile costs about two memory round trips (the pairs, then the gathers)
//      instead of a chain of them;
//   2. stage: the gathered vector entries are fetched and the G products per
//      nonzero written to shared memory;
//   3. sum: a row of at most SEQ_MAX entries is summed by one thread in column
//      order (starting from -0.0 like Rust's `Iterator::sum`, so the FP64 result
//      equals the reference CPU backend's bit for bit); a longer row is summed by
//      one warp (lane-strided partial sums, then a fixed shuffle tree); a row of
//      more than TILE_NNZ entries by the whole CTA (fixed tree);
//   4. epilogue: Op::row() consumes the sums of each row (primal/dual step,
//      Halpern update, residual terms) and may accumulate NP partial sums, which
//      the CTA reduces in a fixed order and writes to per-tile slots.
// Everything is deterministic: the same inputs give the same bits on every run.
#pragma once

#include <map>
#include <mutex>

#include <algorithm>
#include <cstdint>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#include "common.cuh"

namespace sp {

constexpr int NNZ_PER_THREAD = TILE_NNZ / NT;
constexpr int RP_PER_THREAD = (TILE_ROWS + 1 + NT - 1) / NT;
static_assert(TILE_NNZ % NT == 0, "a tile is a whole number of slots per thread");

// Host: cuts rows [0, nrows) into tiles. `rp` has nrows + 1 entries. Tiles that
// hold a single row longer than TILE_NNZ come first so they start early.
inline std::vector<Tile> build_tiles(const int64_t *rp, int64_t nrows) {
    std::vector<Tile> longs, shorts;
    auto tile = [&](int64_t a, int64_t b) { return make_int4((int)a, (int)b, (int)rp[a], (int)rp[b]); };
    int64_t r = 0;
    while (r < nrows) {
        int64_t len = rp[r + 1] - rp[r];
        if (len > TILE_NNZ) {
            longs.push_back(tile(r, r + 1));
            ++r;
            continue;
        }
        int64_t r1 = r, nnz = 0;
        while (r1 < nrows && r1 - r < TILE_ROWS) {
            int64_t l = rp[r1 + 1] - rp[r1];
            if (l > TILE_NNZ || nnz + l > TILE_NNZ) break;
            nnz += l;
            ++r1;
        }
        shorts.push_back(tile(r, r1));
        r = r1;
    }
    longs.insert(longs.end(), shorts.begin(), shorts.end());
    return longs;
}

// Host: the order in which the threads of a tile take its rows (tile-local row
// indices, one uint16 per row, stored at the tile's first row). Rows of at most
// SEQ_MAX entries come first, longest first, dealt so that the 16 rows of every
// half-warp start in 16 different 8-byte shared-memory banks as far as the rows
// allow (the sequential sums then read shared memory without bank conflicts, and
// the rows of a warp have similar lengths); rows summed by a warp come last,
// flagged with SCHED_WARP, so that no warp has to search for them. The schedule
// decides only which thread sums which row, never the order of a row's sum, so
// the rows' results do not depend on it; passes that accumulate partial sums
// across rows do not use it.
constexpr int SCHED_WARP = 0x8000;

inline std::vector<uint16_t> build_schedule(const int64_t *rp, int64_t nrows, const std::vector<Tile> &tiles) {
    std::vector<uint16_t> sched((size_t)std::max<int64_t>(nrows, 0), 0);
    // tiles own disjoint rows: blocks of tiles go to host threads
    auto run = [&](size_t t0, size_t t1) {
        std::vector<int> shortr, heavy, bank, nxt;
        for (size_t ti = t0; ti < t1; ++ti) {
            const Tile &t = tiles[ti];
            const int64_t r0 = t.x, nr = (int64_t)t.y - t.x, k0 = t.z;
            if ((int64_t)t.w - t.z > TILE_NNZ) {  // one long row: the CTA-wide path
                sched[r0] = SCHED_WARP;
                continue;
            }
            // the short rows by decreasing length, ties in row order (a counting sort), and
            // the heavy rows in row order
            int start[SEQ_MAX + 2] = {};
            heavy.clear();
            for (int q = 0; q < nr; ++q) {
                const int64_t len = rp[r0 + q + 1] - rp[r0 + q];
                if (len > SEQ_MAX) heavy.push_back(q);
                else ++start[SEQ_MAX - len + 1];
            }
            for (int l = 1; l <= SEQ_MAX + 1; ++l) start[l] += start[l - 1];
            const int ns = start[SEQ_MAX + 1];
            shortr.resize(ns);
            bank.resize(ns);
            for (int q = 0; q < nr; ++q) {
                const int64_t len = rp[r0 + q + 1] - rp[r0 + q];
                if (len <= SEQ_MAX) shortr[start[SEQ_MAX - len]++] = q;
            }
            for (int c = 0; c < ns; ++c) bank[c] = (int)((rp[r0 + shortr[c]] - k0) & 15);
            // Half-warps of 16 rows in distinct start banks: among the next 64 rows not yet
            // dealt, in sorted order, each whose bank is still free joins; the half-warp is
            // then topped up with the first rows not yet dealt. The rows not yet dealt are a
            // list (nxt, from the head node ns), so each half-warp looks at 64 of them at most.
            nxt.resize(ns + 1);
            for (int c = 0; c < ns; ++c) nxt[c] = c + 1;
            nxt[ns] = ns > 0 ? 0 : ns;
            const int head = ns, end = ns;
            int out = 0;
            while (nxt[head] != end) {
                unsigned mask = 0;
                int placed = 0, seen = 0;
                for (int p = head, c = nxt[head]; c != end && placed < 16 && seen < 64;) {
                    ++seen;
                    if (!((mask >> bank[c]) & 1u)) {
                        mask |= 1u << bank[c];
                        sched[r0 + out++] = (uint16_t)shortr[c];
                        ++placed;
                        nxt[p] = nxt[c];
                        c = nxt[p];
                    } else {
                        p = c;
                        c = nxt[c];
                    }
                }
                while (placed < 16 && nxt[head] != end) {
                    const int c = nxt[head];
                    sched[r0 + out++] = (uint16_t)shortr[c];
                    ++placed;
                    nxt[head] = nxt[c];
                }
            }
            for (size_t i = 0; i < heavy.size(); ++i) sched[r0 + out + i] = (uint16_t)(heavy[i] | SCHED_WARP);
        }
    };
    const size_t nt = tiles.size();
    const int workers = (int)std::min<size_t>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())),
                                              std::max<size_t>(1, nt / 256));
    if (workers <= 1) {
        run(0, nt);
    } else {
        std::vector<std::thread> th;
        for (int w = 0; w < workers; ++w) th.emplace_back(run, nt * w / workers, nt * (w + 1) / workers);
        for (auto &t : th) t.join();
    }
    return sched;
}

// The row schedule of an op, if it carries one.
template <class Op, class = void>
struct has_sched : std::false_type {};
template <class Op>
struct has_sched<Op, std::void_t<decltype(std::declval<Op>().sched)>> : std::true_type {};
template <class Op>
__device__ __forceinline__ const uint16_t *sched_of(const Op &op) {
    if constexpr (has_sched<Op>::value) return op.sched;
    else return nullptr;
}

// Number of leading tiles of a plan that hold a single row longer than TILE_NNZ.
inline int count_long_tiles(const std::vector<Tile> &tiles) {
    int n = 0;
    while (n < (int)tiles.size() && (int64_t)tiles[n].w - tiles[n].z > TILE_NNZ) ++n;
    return n;
}

template <int G, class ST>
constexpr size_t tile_smem_bytes() {
    return (size_t)G * TILE_NNZ * sizeof(ST) + (TILE_ROWS + 1) * sizeof(int);
}

// All G slots' sums of products [a, b) in one walk (slot q in float when bit q of F32 is
// set): each slot is still summed in order from -0.0, but the G chains of adds overlap.
template <int G, unsigned F32, class ST>
__device__ __forceinline__ void seq_sums(const ST *__restrict__ p, int a, int b, double (&s)[G]) {
    float sf[G];
    double sd[G];
#pragma unroll
    for (int q = 0; q < G; ++q) { sf[q] = -0.0f; sd[q] = -0.0; }
    for (int e = a; e < b; ++e) {
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if ((F32 >> q) & 1u) sf[q] += float(p[q * TILE_NNZ + e]);
            else sd[q] += double(p[q * TILE_NNZ + e]);
        }
    }
#pragma unroll
    for (int q = 0; q < G; ++q) s[q] = ((F32 >> q) & 1u) ? double(sf[q]) : sd[q];
}

// The same for a warp row: lane-strided partials of all G slots in one walk, then each
// slot's shuffle tree; lane 0 gets the sums.
template <int G, unsigned F32, class ST>
__device__ __forceinline__ void warp_row_sums(const ST *__restrict__ p, int a, int b, int lane, double (&s)[G]) {
    float sf[G];
    double sd[G];
#pragma unroll
    for (int q = 0; q < G; ++q) { sf[q] = -0.0f; sd[q] = -0.0; }
    for (int e = a + lane; e < b; e += 32) {
#pragma unroll
        for (int q = 0; q < G; ++q) {
            if ((F32 >> q) & 1u) sf[q] += float(p[q * TILE_NNZ + e]);
            else sd[q] += double(p[q * TILE_NNZ + e]);
        }
    }
#pragma unroll
    for (int q = 0; q < G; ++q) s[q] = ((F32 >> q) & 1u) ? double(warp_sum_down(sf[q])) : warp_sum_down(sd[q]);
}

// Streaming loads of the matrix: each element is read once per pass, so they are
// hinted to leave L2 first, which keeps the gathered vectors resident there.
__device__ __forceinline__ int ld_stream(const int *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }

template <class Op>
__device__ __forceinline__ void tile_body(Op &op, unsigned char *smem, int tile) {
    using VT = typename Op::VT;
    using ST = typename Op::ST;
    using Pre = typename Op::Pre;
    constexpr int G = Op::G;
    constexpr int NP = Op::NP;
    constexpr unsigned F32 = Op::F32;  // bit q set: slot q accumulates in float
    ST *prod = reinterpret_cast<ST *>(smem);
    int *srp = reinterpret_cast<int *>(smem + (size_t)G * TILE_NNZ * sizeof(ST));
    const int *__restrict__ rp = op.rp;
    const int *__restrict__ ci = op.ci;
    const VT *__restrict__ vals = op.vals;
    const int tid = threadIdx.x;

    const Tile t = op.tiles[tile];
    const int r0 = t.x, nr = t.y - t.x;
    const int k0 = t.z, nk = t.w - t.z;
    double part[NP > 0 ? NP : 1];
#pragma unroll
    for (int q = 0; q < (NP > 0 ? NP : 1); ++q) part[q] = 0.0;

    if (nk > TILE_NNZ) {
        // One long row: every thread sums a strided slice, then a fixed tree.
        const Pre pre = op.pre(r0);
        float sf[G];
        double sd[G];
#pragma unroll
        for (int q = 0; q < G; ++q) { sf[q] = -0.0f; sd[q] = -0.0; }
        for (int e = tid; e < nk; e += NT) {
            const int k = k0 + e;
            ST p[G];
            op.prod(ld_stream(ci + k), ld_stream(vals + k), p);
#pragma unroll
            for (int q = 0; q < G; ++q) {
                if ((F32 >> q) & 1u) sf[q] += float(p[q]);
                else sd[q] += double(p[q]);
            }
        }
        double *sh = reinterpret_cast<double *>(smem);
        double tot[G];
#pragma unroll
        for (int q = 0; q < G; ++q) {
            // A float slot is reduced in float through the same tree.
            if ((F32 >> q) & 1u) {
                float s = warp_sum_down(sf[q]);
                if ((tid & 31) == 0) sh[tid >> 5] = s;
                __syncthreads();
                if (tid < 32) {
                    float v = tid < NT / 32 ? float(sh[tid]) : 0.0f;
                    v = warp_sum_down(v);
                    tot[q] = v;
                }
                __syncthreads();
            } else {
                double s = warp_sum_down(sd[q]);
                if ((tid & 31) == 0) sh[tid >> 5] = s;
                __syncthreads();
                if (tid < 32) {
                    double v = tid < NT / 32 ? sh[tid] : 0.0;
                    tot[q] = warp_sum_down(v);
                }
                __syncthreads();
            }
        }
        if (tid == 0) op.row(r0, tot, part, pre);
    } else {
        // 1. Issue every load before its first use.
        int rpv[RP_PER_THREAD];
#pragma unroll
        for (int u = 0; u < RP_PER_THREAD; ++u) {
            const int i = tid + u * NT;
            rpv[u] = i <= nr ? rp[r0 + i] : 0;
        }
        // Passes that reduce partial sums keep the row order: the partials a thread
        // accumulates depend on which rows it takes.
        const uint16_t *sched = NP == 0 ? sched_of(op) : nullptr;
        const int e0 = (sched && tid < nr) ? (int)__ldg(sched + r0 + tid) : tid;  // this thread's first slot
        Pre pre{};
        if (tid < nr) pre = op.pre(r0 + (e0 & (SCHED_WARP - 1)));
        int cc[NNZ_PER_THREAD];
        VT vv[NNZ_PER_THREAD];
#pragma unroll
        for (int u = 0; u < NNZ_PER_THREAD; ++u) {
            const int e = tid + u * NT;
            if (e < nk) {
                cc[u] = ld_stream(ci + k0 + e);
                vv[u] = ld_stream(vals + k0 + e);
            }
        }
        // 2. Gathers and products into shared memory.
#pragma unroll
        for (int u = 0; u < NNZ_PER_THREAD; ++u) {
            const int e = tid + u * NT;
            if (e < nk) {
                ST p[G];
                op.prod(cc[u], vv[u], p);
#pragma unroll
                for (int q = 0; q < G; ++q) prod[q * TILE_NNZ + e] = p[q];
            }
        }
#pragma unroll
        for (int u = 0; u < RP_PER_THREAD; ++u) {
            const int i = tid + u * NT;
            if (i <= nr) srp[i] = rpv[u] - k0;
        }
        __syncthreads();
        // 3–4. Short rows: one thread per row, in column order. Thread u takes slot
        // u of the schedule (row u without one).
        for (int u = tid; u < nr; u += NT) {
            const int e = u == tid ? e0 : (sched ? (int)__ldg(sched + r0 + u) : u);
            const int i = e & (SCHED_WARP - 1);
            const int a = srp[i], b = srp[i + 1];
            if (sched ? !(e & SCHED_WARP) : b - a <= SEQ_MAX) {
                double s[G];
                seq_sums<G, F32>(prod, a, b, s);
                if (u == tid) op.row(r0 + i, s, part, pre);
                else op.row(r0 + i, s, part, op.pre(r0 + i));
            }
        }
        // Longer rows: one warp per row (the flagged tail of the schedule).
        const int warp = tid >> 5, lane = tid & 31;
        auto warp_row = [&](int i) {
            const int a = srp[i], b = srp[i + 1];
            double s[G];
            warp_row_sums<G, F32>(prod, a, b, lane, s);
            if (lane == 0) op.row(r0 + i, s, part, op.pre(r0 + i));
        };
        if (sched) {
            for (int u = nr - 1 - warp; u >= 0; u -= NT / 32) {
                const int e = __ldg(sched + r0 + u);
                if (!(e & SCHED_WARP)) break;
                warp_row(e & (SCHED_WARP - 1));
            }
        } else {
            // Rows warp, warp + 8, ... in increasing order, as a scan would take them;
            // a ballot finds the long ones among 32 of them at a time.
            for (int base = warp; base < nr; base += 32 * (NT / 32)) {
                const int i = base + lane * (NT / 32);
                const bool heavy = i < nr && srp[i + 1] - srp[i] > SEQ_MAX;
                for (unsigned mask = __ballot_sync(0xffffffffu, heavy); mask; mask &= mask - 1)
                    warp_row(base + (__ffs(mask) - 1) * (NT / 32));
            }
        }
    }
    if constexpr (NP > 0) {
        __syncthreads();
        block_sum<NP>(part, reinterpret_cast<double *>(smem));
        if (tid == 0) op.store(tile, part);
    }
}

// The tiles of one launch. CTA b takes tile b, then whichever tile is next: ctr[0] counts
// the tiles handed out beyond the first gridDim.x. Tiles are independent and each writes
// its own rows and partial sums, so which CTA takes a tile changes no bit.
template <class Op>
__device__ __forceinline__ void run_tiles(Op &op, unsigned char *smem, int ntiles, int *ctr) {
    __shared__ int next;
    for (int t = blockIdx.x; t < ntiles;) {
        tile_body(op, smem, t);
        __syncthreads();  // the tile is done with shared memory
        if (threadIdx.x == 0) next = (int)gridDim.x + atomicAdd(ctr, 1);
        __syncthreads();
        t = next;
    }
}

// Every CTA of a tile launch ends here, whether or not its pass ran: the last one out
// puts both counters back to zero for the next launch on the stream.
__device__ __forceinline__ void tiles_exit(int *ctr) {
    if (threadIdx.x == 0) {
        __threadfence();  // this CTA's last hand-out before its exit count
        if (atomicAdd(ctr + 1, 1) == (int)gridDim.x - 1) {
            atomicExch(ctr, 0);
            atomicExch(ctr + 1, 0);
        }
    }
}

// One CTA per tile. Op::setup() reads the device state and returns false when the pass
// has nothing to do (solve finished, or a role this epoch skips).
template <class Op>
__global__ void __launch_bounds__(NT) k_tiles(Op op) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (!op.setup()) return;
    tile_body(op, smem, blockIdx.x);
}

// Grid of a persistent tile launch: one CTA per tile, up to as many as the device holds
// at once (then each CTA takes tiles from the launch's counter until none are left). The
// occupancy query is cached per kernel and shared-memory size.
inline unsigned tile_grid(const void *kernel, int sms, int ntiles, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<const void *, size_t>, int> per_sm;
    int bps = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = per_sm.find({kernel, smem});
        if (it != per_sm.end()) {
            bps = it->second;
        } else {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kernel, NT, smem) != cudaSuccess) {
                cudaGetLastError();
                bps = 0;
            }
            per_sm[{kernel, smem}] = bps;
        }
    }
    const int64_t cap = (int64_t)bps * sms;
    return (unsigned)(cap > 0 && cap < ntiles ? cap : ntiles);
}


}  // namespace sp
