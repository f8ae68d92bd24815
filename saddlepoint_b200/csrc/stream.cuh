// stream.cuh — the warp-specialized pipeline of the passes that gather one vector.
//
// The FUSED primal and dual passes (every iteration of an epoch but its first and
// its check) gather a single vector. For them one persistent CTA per SM walks the
// tiles first + blockIdx.x, + gridDim.x, ... through S shared-memory slots with
// three roles that meet only on mbarriers:
//   - a loader (one thread) brings a tile's column indices, values, row pointers,
//     row schedule and the row inputs of its epilogue (x, c, bounds, anchor ...)
//     into a free slot with the bulk copy engine (cp.async.bulk, completion counted
//     on the slot's `load` barrier);
//   - gatherer warps turn the staged column indices into copies of the gathered
//     entries into the slot (register loads, B in flight per lane, then shared
//     stores; or cp.async) and arrive on the slot's `gath` barrier;
//   - eight consumer warps sum the rows of a full slot, run the epilogue and
//     release the slot on its `empty` barrier.
// Each row sum is the tile engine's: products v·g in the op's product type, a row
// of at most SEQ_MAX entries summed by one thread in column order from -0.0, a
// longer one by one warp (lane-strided partials, fixed shuffle tree), a row longer
// than TILE_NNZ (its tile comes first in the plan) by the 256 consumer threads with
// the tile engine's CTA-wide tree. Both engines therefore give the same bits.
//
// Every wait is bounded: a barrier that has not completed after one second (or
// once another role has given up) makes the CTA stop, drain its own copies
// (again bounded) and report through Op::fault().
#pragma once

#include "tiles.cuh"

namespace sp {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One arrival that also announces `bytes` of bulk-copy traffic for this phase.
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr unsigned long long STREAM_WAIT_NS = 1000000000ull;

// Limits of a launch's waits. `withhold` >= 0 is a test knob (set only from the
// SP_TEST_STREAM_WITHHOLD environment variable when a solver is created): the loader
// never issues the copies of that tile, so the roles waiting for it run out of their
// `wait_ns` and take the stall path, with no copy in flight and nothing faulted.
struct StreamTrial {
    unsigned long long wait_ns = STREAM_WAIT_NS;
    int withhold = -1;
};

// Waits for the phase of parity `parity` to complete; false after one second.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > STREAM_WAIT_NS) return false;
    return true;
}

// Bounded wait that also gives up once another role has raised the abort flag.
__device__ __forceinline__ bool stream_wait(unsigned long long *bar, unsigned parity, volatile int *abort,
                                            unsigned long long limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (*abort) return false;
        if (global_ns() - t0 > limit_ns) return false;
    }
    return true;
}

// Bulk copy global -> shared of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) whose completion is counted on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
// Arrives on `bar` once every cp.async this thread has issued so far has landed.
__device__ __forceinline__ void cp_async_mbar_arrive(unsigned long long *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory"); }

// Shape of the CTA: 8 consumer warps (256 threads, the tile engine's NT), one
// loader warp, GW gatherer warps.
constexpr int STREAM_CONSUMER_WARPS = NT / 32;
constexpr int stream_threads(int gw) { return NT + 32 + 32 * gw; }

// Shared memory of one op: S slots of [column indices | values | row pointers |
// gathered entries | row schedule | row inputs], scratch of the long-row tree, 3·S
// mbarriers, the abort flag. Register gatherers (GREG = false) write each product
// v·g over its value, so their slots have no gathered-entry region. SLOTS_DEEP: as many
// slots as fit in the 227 KB a CTA may have (at most 6); otherwise 3 for FP64 ops
// and 4 for FP32 ones, which leaves part of the SM's 256 KB of L1/shared memory to
// the L1 cache that the gathers hit.
constexpr size_t STREAM_SMEM_MAX = 232448;

// Slot modes: SLOTS_FEW (3 FP64 / 4 FP32 slots, one CTA per SM), SLOTS_DEEP (as many as fit,
// one CTA per SM), SLOTS_PAIR (2 slots, two CTAs per SM).
enum : int { SLOTS_FEW = 0, SLOTS_DEEP = 1, SLOTS_PAIR = 2 };
constexpr int stream_ctas_per_sm(int mode) { return mode == SLOTS_PAIR ? 2 : 1; }

template <class Op, bool GREG, int DEEP>
struct StreamLayout {
    using VT = typename Op::VT;
    using GT = typename Op::GT;
    static constexpr int IA = 16 / (int)sizeof(int);       // int32 elements per 16 bytes
    static constexpr int VA = 16 / (int)sizeof(VT);        // value elements per 16 bytes
    static constexpr int DA = 16 / (int)sizeof(double);    // row-input elements per 16 bytes
    static constexpr int SA = 16 / (int)sizeof(uint16_t);  // schedule entries per 16 bytes
    static constexpr size_t up16(size_t b) { return (b + 15) & ~size_t(15); }
    static constexpr size_t ci_bytes = up16(sizeof(int) * (TILE_NNZ + 2 * IA));
    static constexpr size_t v_bytes = up16(sizeof(VT) * (TILE_NNZ + 2 * VA));
    static constexpr size_t rp_bytes = up16(sizeof(int) * (TILE_ROWS + 1 + 2 * IA));
    static constexpr size_t g_bytes = GREG ? up16(sizeof(GT) * TILE_NNZ) : 0;
    static constexpr size_t sch_bytes = up16(sizeof(uint16_t) * (TILE_ROWS + 2 * SA));
    static constexpr int PRE_STRIDE = TILE_ROWS + 2 * DA;  // doubles per row-input array
    static constexpr size_t pre_bytes = sizeof(double) * PRE_STRIDE * Op::NPRE;
    static constexpr size_t ci_off = 0;
    static constexpr size_t v_off = ci_off + ci_bytes;
    static constexpr size_t rp_off = v_off + v_bytes;
    static constexpr size_t g_off = rp_off + rp_bytes;
    static constexpr size_t sch_off = g_off + g_bytes;
    static constexpr size_t pre_off = sch_off + sch_bytes;
    static constexpr size_t slot = pre_off + pre_bytes;
    static constexpr size_t fixed = sizeof(double) * (NT / 32) + 3 * 6 * sizeof(unsigned long long) + 16;
    static constexpr int S_FIT = (int)((STREAM_SMEM_MAX - fixed) / slot) < 6 ? (int)((STREAM_SMEM_MAX - fixed) / slot) : 6;
    static constexpr int S = DEEP == SLOTS_DEEP ? S_FIT : DEEP == SLOTS_PAIR ? 2 : (sizeof(VT) == 4 ? 4 : 3);
    static_assert(S >= 2, "at least two slots");
    static constexpr size_t red_off = S * slot;
    static constexpr size_t bar_off = red_off + sizeof(double) * (NT / 32);
    static constexpr size_t flag_off = bar_off + 3 * 6 * sizeof(unsigned long long);
    static constexpr size_t total = flag_off + 16;
    static_assert(slot % 16 == 0 && (PRE_STRIDE * sizeof(double)) % 16 == 0, "16-byte aligned regions");
};

// Product x of a staged tile: already in place of the value (register gatherers), or
// formed from the value and the gathered entry (cp.async gatherers).
template <bool IN_PLACE, class Op>
__device__ __forceinline__ typename Op::ST prod_at(const Op &op, const typename Op::VT *vs, const typename Op::GT *gs,
                                                   int x) {
    if constexpr (IN_PLACE) return reinterpret_cast<const typename Op::ST *>(vs)[x];
    else return op.mul(vs[x], gs[x]);
}

template <class Op>
__device__ __forceinline__ void stream_abort(const Op &op, int *abort) {
    if (atomicExch(abort, 1) == 0) op.fault();
}

// A row longer than TILE_NNZ, summed by the 256 consumer threads exactly as
// tile_body sums it: thread t takes entries t, t+NT, ... in order (eight loads in
// flight at a time), then a shuffle tree per warp and one over the warp totals.
template <class Op>
__device__ __forceinline__ void consumer_long_row(Op &op, double *sh, int tile) {
    using VT = typename Op::VT;
    using ST = typename Op::ST;
    constexpr bool F32 = (Op::F32 & 1u) != 0;
    const int tid = threadIdx.x;
    const Tile t = op.tiles[tile];
    const int r0 = t.x, k0 = t.z, nk = t.w - t.z;
    const typename Op::Pre pre = op.pre(r0);
    float sf = -0.0f;
    double sd = -0.0;
    for (int base = tid; base < nk; base += 8 * NT) {
        int c[8];
        VT v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * NT;
            if (e < nk) {
                c[u] = ld_stream(op.ci + k0 + e);
                v[u] = ld_stream(op.vals + k0 + e);
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            if (base + u * NT < nk) {
                ST p[1];
                op.prod(c[u], v[u], p);
                if constexpr (F32) sf += float(p[0]);
                else sd += double(p[0]);
            }
        }
    }
    double tot[1] = {0.0};
    if constexpr (F32) {
        const float s = warp_sum_down(sf);
        if ((tid & 31) == 0) sh[tid >> 5] = s;
        consumer_sync();
        if (tid < 32) {
            float v = tid < NT / 32 ? float(sh[tid]) : 0.0f;
            tot[0] = warp_sum_down(v);
        }
    } else {
        const double s = warp_sum_down(sd);
        if ((tid & 31) == 0) sh[tid >> 5] = s;
        consumer_sync();
        if (tid < 32) {
            double v = tid < NT / 32 ? sh[tid] : 0.0;
            tot[0] = warp_sum_down(v);
        }
    }
    consumer_sync();
    double part[1] = {0.0};
    if (tid == 0) op.row(r0, tot, part, pre);
}

// GW gatherer warps; LDG: gathers through registers (B loads in flight per lane,
// then the products stored over the values and a plain arrive) instead of cp.async;
// DEEP: the slot count (StreamLayout).
template <int GW, bool LDG, int B, int DEEP, class Op>
__device__ __forceinline__ void stream_run(Op &op, unsigned char *smem, int ntiles, int nlong, const StreamTrial tr) {
    using VT = typename Op::VT;
    using GT = typename Op::GT;
    using ST = typename Op::ST;
    using L = StreamLayout<Op, !LDG, DEEP>;
    constexpr int S = L::S;
    static_assert(Op::G == 1 && Op::NP == 0, "the stream engine runs passes that gather one vector and reduce nothing");
    static_assert(!LDG || sizeof(ST) == sizeof(VT), "a product takes its value's place");
    constexpr bool F32 = (Op::F32 & 1u) != 0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long *bar_load = reinterpret_cast<unsigned long long *>(smem + L::bar_off);
    unsigned long long *bar_gath = bar_load + S;
    unsigned long long *bar_empty = bar_gath + S;
    int *abort = reinterpret_cast<int *>(smem + L::flag_off);
    volatile int *abort_v = abort;

    const int first = nlong + blockIdx.x, step = gridDim.x;
    const int nmine = first < ntiles ? (ntiles - first + step - 1) / step : 0;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(bar_load + s, 1);
            mbar_init(bar_gath + s, 32 * GW);
            mbar_init(bar_empty + s, STREAM_CONSUMER_WARPS);
        }
        *abort = 0;
        mbar_init_fence();
    }
    __syncthreads();

    if (warp == STREAM_CONSUMER_WARPS) {
        // ---- loader ----
        if (lane != 0) return;
        unsigned pend = 0, par = 0;  // slots with a copy outstanding and its phase parity
        for (int j = 0; j < nmine; ++j) {
            const int s = j % S, k = j / S;
            if (k >= 1 && !stream_wait(bar_empty + s, (unsigned)(k - 1) & 1u, abort_v, tr.wait_ns)) {
                stream_abort(op, abort);
                break;
            }
            if (first + j * step == tr.withhold) continue;  // test knob: no copy, no arrival
            const Tile t = op.tiles[first + j * step];
            const int ka = t.z & ~(L::IA - 1), kb = (t.w + L::IA - 1) & ~(L::IA - 1);
            const int va = t.z & ~(L::VA - 1), vb = (t.w + L::VA - 1) & ~(L::VA - 1);
            const int ra = t.x & ~(L::IA - 1), rb = (t.y + 1 + L::IA - 1) & ~(L::IA - 1);
            const int pa = t.x & ~(L::DA - 1), pb = (t.y + L::DA - 1) & ~(L::DA - 1);
            const int sa = t.x & ~(L::SA - 1), sb = (t.y + L::SA - 1) & ~(L::SA - 1);
            const unsigned bc = (unsigned)(kb - ka) * 4u, bv = (unsigned)(vb - va) * (unsigned)sizeof(VT);
            const unsigned br = (unsigned)(rb - ra) * 4u, bp = (unsigned)(pb - pa) * 8u;
            const unsigned bs = (unsigned)(sb - sa) * (unsigned)sizeof(uint16_t);
            unsigned char *slot = smem + s * L::slot;
            unsigned long long *bar = bar_load + s;
            mbar_expect_tx(bar, bc + bv + br + bs + bp * Op::NPRE);
            if (bc) bulk_g2s(slot + L::ci_off, op.ci + ka, bc, bar);
            if (bv) bulk_g2s(slot + L::v_off, op.vals + va, bv, bar);
            bulk_g2s(slot + L::rp_off, op.rp + ra, br, bar);
            bulk_g2s(slot + L::sch_off, op.sched + sa, bs, bar);
            for (int q = 0; q < Op::NPRE; ++q)
                bulk_g2s(slot + L::pre_off + (size_t)q * L::PRE_STRIDE * sizeof(double), op.pre_array(q) + pa, bp,
                         bar);
            pend |= 1u << s;
            par = (par & ~(1u << s)) | ((unsigned)(k & 1) << s);
        }
        // Every copy this thread started lands before the CTA may end.
        for (int s = 0; s < S; ++s)
            if (pend & (1u << s)) (void)mbar_wait(bar_load + s, (par >> s) & 1u);
        return;
    }
    if (warp > STREAM_CONSUMER_WARPS) {
        // ---- gatherers ----
        const int g = warp - STREAM_CONSUMER_WARPS - 1;
        const GT *__restrict__ gv = op.gvec();
        for (int j = 0; j < nmine; ++j) {
            const int s = j % S, k = j / S;
            if (!stream_wait(bar_load + s, (unsigned)k & 1u, abort_v, tr.wait_ns)) {
                stream_abort(op, abort);
                break;
            }
            const Tile t = op.tiles[first + j * step];
            const int nk = t.w - t.z;
            const unsigned char *slot = smem + s * L::slot;
            const int *cs = reinterpret_cast<const int *>(slot + L::ci_off) + (t.z & (L::IA - 1));
            GT *gs = reinterpret_cast<GT *>(smem + s * L::slot + L::g_off);
            if constexpr (LDG) {
                // the product v·g replaces the staged value (one shared array for the sums)
                ST *ps = reinterpret_cast<ST *>(smem + s * L::slot + L::v_off) + (t.z & (L::VA - 1));
                constexpr int W = 32 * GW;
                for (int base = g * 32 + lane; base < nk; base += W * B) {
                    GT v[B];
#pragma unroll
                    for (int u = 0; u < B; ++u)
                        if (base + u * W < nk) v[u] = __ldg(gv + cs[base + u * W]);
#pragma unroll
                    for (int u = 0; u < B; ++u)
                        if (base + u * W < nk) {
                            const int e = base + u * W;
                            ps[e] = op.mul(reinterpret_cast<const VT *>(ps)[e], v[u]);
                        }
                }
                mbar_arrive(bar_gath + s);  // release: the stores above are visible to the waiters
            } else {
                for (int e = g * 32 + lane; e < nk; e += 32 * GW) cp_async<(int)sizeof(GT)>(gs + e, gv + cs[e]);
                cp_async_mbar_arrive(bar_gath + s);
            }
        }
        if constexpr (!LDG) cp_async_wait_all();
        return;
    }

    // ---- consumers (threads 0..255) ----
    const int tid = threadIdx.x;
    for (int t = blockIdx.x; t < nlong; t += gridDim.x) {
        consumer_long_row(op, reinterpret_cast<double *>(smem + L::red_off), t);
        consumer_sync();
    }
    double part[1] = {0.0};
    for (int j = 0; j < nmine; ++j) {
        const int s = j % S, k = j / S;
        if (!stream_wait(bar_load + s, (unsigned)k & 1u, abort_v, tr.wait_ns) ||
            !stream_wait(bar_gath + s, (unsigned)k & 1u, abort_v, tr.wait_ns)) {
            stream_abort(op, abort);
            break;
        }
        const Tile t = op.tiles[first + j * step];
        const int r0 = t.x, nr = t.y - t.x, k0 = t.z;
        const unsigned char *slot = smem + s * L::slot;
        const VT *vs = reinterpret_cast<const VT *>(slot + L::v_off) + (k0 & (L::VA - 1));
        const int *rps = reinterpret_cast<const int *>(slot + L::rp_off) + (r0 & (L::IA - 1));
        const GT *gs = reinterpret_cast<const GT *>(slot + L::g_off);
        const uint16_t *ss = reinterpret_cast<const uint16_t *>(slot + L::sch_off) + (r0 & (L::SA - 1));
        const double *pres = reinterpret_cast<const double *>(slot + L::pre_off) + (r0 & (L::DA - 1));
        // Schedule slots are dealt to threads (and the flagged tail to warps) with an
        // offset that rotates per tile by whole warps, so short tiles do not always
        // land on the same warps.
        const int rot = j & 7;
        for (int u = (tid + 32 * rot) & (NT - 1); u < nr; u += NT) {
            const int e = ss[u];
            if (e & SCHED_WARP) continue;
            const int q = e;
            const int a = rps[q] - k0, b = rps[q + 1] - k0;
            double sum[1];
            if constexpr (F32) {
                float f = -0.0f;
                for (int x = a; x < b; ++x) f += float(prod_at<LDG>(op, vs, gs, x));
                sum[0] = double(f);
            } else {
                double d = -0.0;
                for (int x = a; x < b; ++x) d += double(prod_at<LDG>(op, vs, gs, x));
                sum[0] = d;
            }
            op.row(r0 + q, sum, part, op.pre_smem(pres + q, L::PRE_STRIDE));
        }
        for (int u = nr - 1 - ((warp + rot) & 7); u >= 0; u -= NT / 32) {
            const int e = ss[u];
            if (!(e & SCHED_WARP)) break;
            const int q = e & (SCHED_WARP - 1);
            const int a = rps[q] - k0, b = rps[q + 1] - k0;
            double sum[1];
            if constexpr (F32) {
                float f = -0.0f;
                for (int x = a + lane; x < b; x += 32) f += float(prod_at<LDG>(op, vs, gs, x));
                sum[0] = double(warp_sum_down(f));
            } else {
                double d = -0.0;
                for (int x = a + lane; x < b; x += 32) d += double(prod_at<LDG>(op, vs, gs, x));
                sum[0] = warp_sum_down(d);
            }
            if (lane == 0) op.row(r0 + q, sum, part, op.pre_smem(pres + q, L::PRE_STRIDE));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(bar_empty + s);
    }
}

// Runs the pass `op` if its setup() accepts this launch (a uniform choice: it
// depends only on the device state). One CTA of stream_threads(GW) per SM, with
// StreamLayout<Op, !LDG, DEEP>::total bytes of dynamic shared memory.
template <class Op, int GW, bool LDG, int B, int DEEP>
__global__ void __launch_bounds__(stream_threads(GW), stream_ctas_per_sm(DEEP)) k_stream(int ntiles, int nlong, Op op, StreamTrial tr) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (op.setup()) stream_run<GW, LDG, B, DEEP>(op, smem, ntiles, nlong, tr);
}

}  // namespace sp
