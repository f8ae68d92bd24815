// batch.cu — the batched form (Part 3 of the C ABI).
//
// sp_batch_create packs every LP into one arena (int32 instance-local row
// pointers, column indices, values, vectors), builds each A'ᵀ on the host with the
// reference's stable counting sort (problem.rs:88-109, bit for bit), picks the
// lanes-per-row SpMV variant of every instance with the tuner below, and captures
// [reset the work counter, launch the persistent kernel] as one CUDA graph.
// sp_batch_solve replays the graph; the scaling, power iteration and PDHG loop of
// every instance run inside the kernel (batch_kernels.cuh).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "batch_kernels.cuh"
#include "internal.cuh"

struct sp_batch {
    sp_ctx *ctx = nullptr;
    int count = 0;
    int mixed = 0;
    int64_t total_m = 0, total_n = 0, total_nnz = 0;
    std::vector<sp::BatchInst> inst;
    sp::BatchArgs args{};
    std::vector<void *> bufs;
    cudaGraphExec_t graph = nullptr;
    int grid = 0;
    sp::BatchInst *d_inst = nullptr;
    int *d_counter = nullptr;
    double *av0 = nullptr, *tv0 = nullptr;  // the original values (the kernel scales in place)
    size_t smem = 0;
    double tuned_us[4][8] = {};  // per-iteration µs of each tuned shape at the calibration sizes
    int tuned_nnz[8] = {};
    int tuned_points = 0;
    sp_solver_params params{};  // every instance's parameters (the hand-off solves use them too)
};

namespace sp {

// Lanes per row for a matrix whose rows hold `mean` entries on average: the
// smallest power of two that leaves each lane about `per_lane` products (one lane per
// row keeps the reference's summation order for short rows).
int lanes_for(double mean, int per_lane = 3) {
    int L = 1;
    while (L < 32 && L * per_lane < mean) L <<= 1;
    return L;
}

// The shapes the tuner times: lane groups with about 3, 2 or 6 products per lane, and the
// staged tiles.
constexpr int TUNE_SHAPES = 4;
constexpr int SHAPE_TILES = 1;
int shape_per_lane(int shape) { return shape == 2 ? 2 : shape == 3 ? 6 : 3; }

// Gives instance I the SpMV shape `shape` (its variant and lanes per row).
void apply_shape(BatchInst &I, int shape) {
    I.variant = shape == SHAPE_TILES ? VARIANT_TILES : VARIANT_LANES;
    const int k = shape_per_lane(shape);
    I.lanes_a = lanes_for(I.m ? (double)I.nnz / I.m : 0.0, k);
    I.lanes_t = lanes_for(I.n ? (double)I.nnz / I.n : 0.0, k);
}

template <class T>
int balloc(sp_batch *b, T **p, int64_t n) {
    SP_CUDA_TRY(cudaMalloc(p, sizeof(T) * std::max<int64_t>(n, 1)));
    b->bufs.push_back(*p);
    return SP_OK;
}

// The autotuner. Once per device it times four SpMV shapes — lane groups (rows dealt to
// L lanes that walk them with strided loads, L the smallest power of two leaving each
// lane about 3, 2 or 6 products) and staged tiles (the single-LP tile passes) — on
// built-in seeded reference LPs that span the sizes of the batched workload, each alone
// in one CTA, as the difference of a 320- and a 64-iteration run (the scaling passes and
// the power iteration cancel). Every instance then gets the shape whose interpolated
// per-iteration time at its size (log nnz) is lowest, with its own L from its mean row
// lengths. The choice depends on the instance alone, never on the rest
// of the batch, so an instance is computed the same way alone and in any mix.
// SP_BATCH_VARIANT=lanes|tiles in the environment forces one variant.
struct TuneTable {
    bool ready = false;
    int npts = 0;
    int nnz[8] = {};
    double us[TUNE_SHAPES][8] = {};
};
static TuneTable g_tune[64];
static std::mutex g_tune_mu;

int batch_create(sp_ctx *ctx, const sp_lp *lps, int count, const sp_solver_params *params, sp_batch **out,
                 bool tune);

int calibrate(sp_ctx *ctx, TuneTable *T) {
    // reference LPs: the random LP recipe, m from 60 to 2000, n = 2m, 3-8 nonzeros per column
    const int ms[] = {60, 180, 540, 2000};
    std::vector<sp_lp> lps;
    int rc = SP_OK;
    for (int q = 0; q < 4 && !rc; ++q) {
        sp_gen_params g{};
        g.kind = SP_GEN_RANDOM;
        g.seed = 0x5EED0000u + q;
        g.nrows = ms[q];
        g.ncols = 2 * ms[q];
        g.nnz_per_col_min = 3;
        g.nnz_per_col_max = 8;
        sp_lp lp{};
        rc = sp_generate(&g, &lp);
        if (!rc) lps.push_back(lp);
    }
    sp_batch *b = nullptr;
    if (!rc) rc = batch_create(ctx, lps.data(), (int)lps.size(), nullptr, &b, false);
    if (!rc) {
        cudaStream_t st = ctx->stream;
        std::vector<BatchInst> &inst = b->inst;
        int *d_one = nullptr;
        rc = balloc(b, &d_one, 1);
        BatchArgs A2 = b->args;
        A2.count = 1;
        A2.order = d_one;
        A2.base.tolerance = 0.0;  // never converged: every run takes exactly its iterations
        A2.handoff_ns = 0;
        A2.power_iterations = std::min<unsigned long long>(A2.power_iterations, 4);
        EventPair ep;
        if (!rc) rc = ep.init();
        cudaEvent_t e0 = ep.e0, e1 = ep.e1;
        auto run = [&](int c, unsigned long long iters, float *ms_out) -> int {
            const BatchInst &I = inst[c];
            A2.base.max_iterations = iters;
            SP_CUDA_TRY(cudaMemcpyAsync(d_one, &c, sizeof(int), cudaMemcpyHostToDevice, st));
            SP_CUDA_TRY(cudaMemcpyAsync(b->args.a_v + I.nz, b->av0 + I.nz, sizeof(double) * I.nnz,
                                        cudaMemcpyDeviceToDevice, st));
            SP_CUDA_TRY(cudaMemcpyAsync(b->args.t_v + I.nz, b->tv0 + I.nz, sizeof(double) * I.nnz,
                                        cudaMemcpyDeviceToDevice, st));
            SP_CUDA_TRY(cudaMemsetAsync(b->d_counter, 0, sizeof(int), st));
            SP_CUDA_TRY(cudaEventRecord(e0, st));
            k_batch<NT><<<1, NT, b->smem, st>>>(A2);
            SP_CUDA_TRY(cudaEventRecord(e1, st));
            SP_CUDA_TRY(cudaEventSynchronize(e1));
            SP_CUDA_TRY(cudaEventElapsedTime(ms_out, e0, e1));
            return SP_OK;
        };
        const int npts = (int)inst.size();
        for (int v = 0; v < TUNE_SHAPES && !rc; ++v) {
            for (auto &I : inst) apply_shape(I, v);
            rc = cudaMemcpy(b->d_inst, inst.data(), sizeof(BatchInst) * npts, cudaMemcpyHostToDevice) == cudaSuccess
                     ? SP_OK
                     : SP_ERR_CUDA;
            for (int p = 0; p < npts && !rc; ++p) {
                float t1 = 0, t2 = 0;
                if ((rc = run(p, 64, &t1)) || (rc = run(p, 320, &t2))) break;
                T->us[v][p] = std::max(0.0, (double)(t2 - t1) * 1e3 / 256.0);
                T->nnz[p] = inst[p].nnz;
            }
        }
        T->npts = npts;
        T->ready = rc == SP_OK;
    }
    if (b) sp_batch_free(b);
    for (auto &lp : lps) sp_lp_release(&lp);
    return rc;
}

int tune_variants(sp_batch *b) {
    std::vector<BatchInst> &inst = b->inst;
    int forced = -1;
    if (const char *env = getenv("SP_BATCH_VARIANT"))
        forced = !strcmp(env, "lanes") ? VARIANT_LANES : (!strcmp(env, "tiles") ? VARIANT_TILES : -1);
    if (forced < 0) {
        const int dev = b->ctx->device;
        std::lock_guard<std::mutex> lock(g_tune_mu);
        if (dev < 0 || dev >= 64) return SP_ERR_INVALID;
        if (!g_tune[dev].ready) {
            int rc = calibrate(b->ctx, &g_tune[dev]);
            if (rc) return rc;
            set_current_ctx(b->ctx);
        }
        const TuneTable &T = g_tune[dev];
        b->tuned_points = T.npts;
        for (int p = 0; p < T.npts; ++p) {
            b->tuned_nnz[p] = T.nnz[p];
            for (int v = 0; v < TUNE_SHAPES; ++v) b->tuned_us[v][p] = T.us[v][p];
        }
        auto estimate = [&](int v, int nnz) {
            const double x = std::log(std::max(1, nnz));
            if (T.npts == 1) return T.us[v][0];
            int p = 0;
            while (p + 2 < T.npts && std::log(std::max(1, T.nnz[p + 1])) < x) ++p;
            const double x0 = std::log(std::max(1, T.nnz[p])), x1 = std::log(std::max(1, T.nnz[p + 1]));
            const double f = x1 > x0 ? std::min(1.0, std::max(0.0, (x - x0) / (x1 - x0))) : 0.0;
            return T.us[v][p] + f * (T.us[v][p + 1] - T.us[v][p]);
        };
        for (auto &I : inst) {
            int best = 0;
            for (int v = 1; v < TUNE_SHAPES; ++v)
                if (estimate(v, I.nnz) < estimate(best, I.nnz)) best = v;
            apply_shape(I, best);
        }
    } else {
        for (auto &I : inst) apply_shape(I, forced == VARIANT_TILES ? SHAPE_TILES : 0);
    }
    cudaStream_t st = b->ctx->stream;
    SP_CUDA_TRY(cudaMemcpyAsync(b->d_inst, inst.data(), sizeof(BatchInst) * b->count, cudaMemcpyHostToDevice, st));
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    return SP_OK;
}

// The instance as an sp_lp again, from the arena's original data on the device.
struct HostLp {
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v, c, lc, uc, lv, uv;
    sp_lp lp{};
};

int download_instance(const sp_batch *b, int i, HostLp *h) {
    const BatchInst &I = b->inst[i];
    const BatchArgs &A = b->args;
    std::vector<int> rp32(I.m + 1);
    h->ci.resize(std::max(I.nnz, 1));
    h->v.resize(std::max(I.nnz, 1));
    h->c.resize(std::max(I.n, 1));
    h->lv.resize(std::max(I.n, 1));
    h->uv.resize(std::max(I.n, 1));
    h->lc.resize(std::max(I.m, 1));
    h->uc.resize(std::max(I.m, 1));
    auto get = [](void *dst, const void *src, size_t bytes) -> int {
        if (bytes) SP_CUDA_TRY(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
        return SP_OK;
    };
    int rc;
    if ((rc = get(rp32.data(), A.a_rp + I.rpa, sizeof(int) * (I.m + 1))) ||
        (rc = get(h->ci.data(), A.a_ci + I.nz, sizeof(int) * I.nnz)) ||
        (rc = get(h->v.data(), b->av0 + I.nz, sizeof(double) * I.nnz)) ||
        (rc = get(h->c.data(), A.oc + I.no, sizeof(double) * I.n)) ||
        (rc = get(h->lv.data(), A.olv + I.no, sizeof(double) * I.n)) ||
        (rc = get(h->uv.data(), A.ouv + I.no, sizeof(double) * I.n)) ||
        (rc = get(h->lc.data(), A.olc + I.mo, sizeof(double) * I.m)) ||
        (rc = get(h->uc.data(), A.ouc + I.mo, sizeof(double) * I.m)))
        return rc;
    h->rp.assign(rp32.begin(), rp32.end());
    sp_lp &L = h->lp;
    L.a.nrows = I.m;
    L.a.ncols = I.n;
    L.a.nnz = I.nnz;
    L.a.row_ptr = h->rp.data();
    L.a.col_idx = h->ci.data();
    L.a.values = h->v.data();
    L.c = h->c.data();
    L.lc = h->lc.data();
    L.uc = h->uc.data();
    L.lv = h->lv.data();
    L.uv = h->uv.data();
    L.c0 = I.c0;
    L.maximize = I.maximize;
    return SP_OK;
}

// Solves the instances the kernel stopped for the hand-off again with sp_solve,
// up to eight at a time, each on a context (stream) of its own, and writes their
// results and solutions where the kernel's would have gone.
int hand_off(sp_batch *b, std::vector<sp_batch_result> &res) {
    std::vector<int> todo;
    for (int i = 0; i < b->count; ++i)
        if (res[i].handed_off == 2) todo.push_back(i);
    if (todo.empty()) return SP_OK;
    // the largest first, so the longest solves start early
    std::stable_sort(todo.begin(), todo.end(), [&](int a, int c) { return b->inst[a].nnz > b->inst[c].nnz; });
    const int workers = (int)std::min<size_t>(8, todo.size());
    std::atomic<size_t> next{0};
    std::mutex mu;
    int first_err = SP_OK;
    std::string err_msg;
    auto work = [&]() {
        sp_ctx *ctx = nullptr;
        int rc = sp_ctx_create(b->ctx->device, &ctx);
        size_t k;
        while (!rc && (k = next.fetch_add(1)) < todo.size()) {
            const int i = todo[k];
            const BatchInst &I = b->inst[i];
            HostLp h;
            std::vector<double> x(std::max(I.n, 1)), y(std::max(I.m, 1));
            sp_solution_info info{};
            if ((rc = download_instance(b, i, &h))) break;
            sp_batch_result &r = res[i];
            rc = sp_solve(ctx, &h.lp, &b->params, x.data(), y.data(), &info);
            if (rc == SP_ERR_NUMERICAL) {
                // a breakdown is this instance's result, as the kernel reports it
                const bool power = ctx->last_error.find("power") != std::string::npos;
                r.status = -1 - (power ? ERR_NUMERICAL_POWER : ERR_NUMERICAL_ITERATES);
                r.handed_off = 1;
                rc = SP_OK;
                continue;
            }
            if (rc) break;
            if (I.n && cudaMemcpy(b->args.ox + I.no, x.data(), sizeof(double) * I.n, cudaMemcpyHostToDevice))
                rc = SP_ERR_CUDA;
            if (I.m && cudaMemcpy(b->args.oy + I.mo, y.data(), sizeof(double) * I.m, cudaMemcpyHostToDevice))
                rc = SP_ERR_CUDA;
            r.status = info.status;
            r.objective = info.objective;
            r.dual_objective = info.dual_objective;
            r.primal_residual = info.primal_residual;
            r.dual_residual = info.dual_residual;
            r.gap = info.gap;
            r.iterations = info.iterations;
            r.restarts = info.restarts;
            r.handed_off = 1;
        }
        if (rc) {
            std::lock_guard<std::mutex> lock(mu);
            if (!first_err) {
                first_err = rc;
                err_msg = ctx ? ctx->last_error : std::string("sp_ctx_create failed");
            }
        }
        if (ctx) sp_ctx_destroy(ctx);
    };
    std::vector<std::thread> th;
    for (int w = 0; w < workers; ++w) th.emplace_back(work);
    for (auto &t : th) t.join();
    set_current_ctx(b->ctx);
    SP_CUDA_TRY(cudaSetDevice(b->ctx->device));
    if (first_err) return fail(first_err, "batch hand-off solve: " + err_msg);
    return SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" void sp_batch_free(sp_batch *b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (void *p : b->bufs) cudaFree(p);
    delete b;
}

extern "C" int sp_batch_create(sp_ctx *ctx, const sp_lp *lps, int count, const sp_solver_params *params,
                               sp_batch **out) {
    int rc = enter(ctx);
    if (rc) return rc;
    return batch_create(ctx, lps, count, params, out, true);
}

namespace sp {
int batch_create(sp_ctx *ctx, const sp_lp *lps, int count, const sp_solver_params *params, sp_batch **out,
                 bool tune) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!lps || count <= 0 || !out) return fail(SP_ERR_INVALID, "sp_batch_create: bad arguments");
    for (int i = 0; i < count; ++i) {  // each instance as Solver::new validates it (solver.rs:155)
        char msg[256] = "";
        const int v = sp_problem_validate(&lps[i], msg, sizeof msg);
        if (v != SP_OK) return fail(v, "instance " + std::to_string(i) + ": " + (msg[0] ? msg : "lacks an array"));
    }
    sp_solver_params P;
    sp_solver_params_default(&P);
    if (params) P = *params;
    auto *b = new sp_batch();
    b->ctx = ctx;
    b->count = count;
    b->params = P;
    b->mixed = P.precision == SP_PRECISION_MIXED;
    auto bail = [&](int code, const std::string &msg) {
        sp_batch_free(b);
        return fail(code, msg);
    };
    // offsets
    b->inst.resize(count);
    int64_t rpa = 0, rpt = 0, nz = 0, mo = 0, no = 0;
    for (int i = 0; i < count; ++i) {
        const sp_lp &L = lps[i];
        const sp_csr &A = L.a;
        if (A.nrows < 0 || A.ncols < 0 || A.nnz < 0 || !A.row_ptr || A.row_ptr[A.nrows] != A.nnz)
            return bail(SP_ERR_INVALID, "sp_batch_create: bad CSR");
        for (int64_t j = 0; j < A.ncols; ++j)
            if (std::isnan(L.lv[j]) || std::isnan(L.uv[j]) || L.lv[j] > L.uv[j] || std::isnan(L.c[j]))
                return bail(SP_ERR_PROBLEM, "sp_batch_create: invalid variable bounds or cost");
        for (int64_t r = 0; r < A.nrows; ++r)
            if (std::isnan(L.lc[r]) || std::isnan(L.uc[r]) || L.lc[r] > L.uc[r])
                return bail(SP_ERR_PROBLEM, "sp_batch_create: invalid constraint bounds");
        BatchInst &I = b->inst[i];
        I = BatchInst{};
        I.m = (int)A.nrows;
        I.n = (int)A.ncols;
        I.nnz = (int)A.nnz;
        apply_shape(I, 0);
        I.rpa = rpa;
        I.rpt = rpt;
        I.nz = nz;
        I.mo = mo;
        I.no = no;
        I.c0 = L.c0;
        I.maximize = L.maximize;
        rpa += A.nrows + 1;
        rpt += A.ncols + 1;
        nz += A.nnz;
        mo += A.nrows;
        no += A.ncols;
    }
    if (nz > INT32_MAX || rpa > INT32_MAX || rpt > INT32_MAX)
        return bail(SP_ERR_TOO_LARGE, "batch too large for 32-bit indices");
    b->total_m = mo;
    b->total_n = no;
    b->total_nnz = nz;
    // host arena, transposes built in parallel (each instance's own counting sort)
    std::vector<int> h_arp(rpa), h_trp(rpt), h_aci(std::max<int64_t>(nz, 1)), h_tci(std::max<int64_t>(nz, 1));
    std::vector<double> h_av(std::max<int64_t>(nz, 1)), h_tv(std::max<int64_t>(nz, 1));
    std::vector<double> h_c(no), h_lv(no), h_uv(no), h_lc(mo), h_uc(mo);
    auto pack = [&](int i0, int i1) {
        for (int i = i0; i < i1; ++i) {
            const sp_lp &L = lps[i];
            const BatchInst &I = b->inst[i];
            const int m = I.m, n = I.n;
            for (int r = 0; r <= m; ++r) h_arp[I.rpa + r] = (int)L.a.row_ptr[r];
            std::copy(L.a.col_idx, L.a.col_idx + I.nnz, h_aci.begin() + I.nz);
            std::copy(L.a.values, L.a.values + I.nnz, h_av.begin() + I.nz);
            std::copy(L.c, L.c + n, h_c.begin() + I.no);
            std::copy(L.lv, L.lv + n, h_lv.begin() + I.no);
            std::copy(L.uv, L.uv + n, h_uv.begin() + I.no);
            std::copy(L.lc, L.lc + m, h_lc.begin() + I.mo);
            std::copy(L.uc, L.uc + m, h_uc.begin() + I.mo);
            // CsrMatrix::transpose (problem.rs:88-109)
            int *cnt = &h_trp[I.rpt];
            std::fill(cnt, cnt + n + 1, 0);
            for (int k = 0; k < I.nnz; ++k) cnt[L.a.col_idx[k] + 1] += 1;
            for (int j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
            std::vector<int> next(cnt, cnt + n);
            for (int r = 0; r < m; ++r)
                for (int64_t k = L.a.row_ptr[r]; k < L.a.row_ptr[r + 1]; ++k) {
                    const int t = next[L.a.col_idx[k]]++;
                    h_tci[I.nz + t] = r;
                    h_tv[I.nz + t] = L.a.values[k];
                }
        }
    };
    {
        int nt = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(pack, count * t / nt, count * (t + 1) / nt);
        for (auto &t : th) t.join();
    }
    // tile plans of every instance (tiles.cuh), for the tile variant
    std::vector<std::vector<Tile>> tiles_a(count), tiles_t(count);
    auto plan = [&](int i0, int i1) {
        std::vector<int64_t> rp;
        for (int i = i0; i < i1; ++i) {
            const BatchInst &I = b->inst[i];
            rp.assign(h_arp.begin() + I.rpa, h_arp.begin() + I.rpa + I.m + 1);
            tiles_a[i] = build_tiles(rp.data(), I.m);
            rp.assign(h_trp.begin() + I.rpt, h_trp.begin() + I.rpt + I.n + 1);
            tiles_t[i] = build_tiles(rp.data(), I.n);
        }
    };
    {
        int nt = std::max(1, std::min<int>(16, (int)std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(plan, count * t / nt, count * (t + 1) / nt);
        for (auto &t : th) t.join();
    }
    int64_t n_ta = 0, n_tt = 0, n_part = 0;
    for (int i = 0; i < count; ++i) {
        BatchInst &I = b->inst[i];
        I.ta = n_ta;
        I.nta = (int)tiles_a[i].size();
        n_ta += I.nta;
        I.tt = n_tt;
        I.ntt = (int)tiles_t[i].size();
        n_tt += I.ntt;
        I.pa = n_part;
        n_part += (int64_t)I.nta * (NP_D + NP_D0);
        I.pt = n_part;
        n_part += (int64_t)I.ntt * (NP_P + NP_T + NP_P0 + 1);
        I.variant = VARIANT_TILES;
    }
    std::vector<Tile> h_ta(std::max<int64_t>(n_ta, 1)), h_tt(std::max<int64_t>(n_tt, 1));
    for (int i = 0; i < count; ++i) {
        std::copy(tiles_a[i].begin(), tiles_a[i].end(), h_ta.begin() + b->inst[i].ta);
        std::copy(tiles_t[i].begin(), tiles_t[i].end(), h_tt.begin() + b->inst[i].tt);
    }
    // processing order: largest first, so the long instances start early
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->inst[a].nnz > b->inst[c].nnz; });

    BatchArgs &A = b->args;
    A.count = count;
    A.mixed = b->mixed;
    BatchInst *d_inst;
    int *d_order, *d_counter, *arp, *aci, *trp, *tci;
    double *av, *tv, *oc, *olv, *ouv, *olc, *ouc;
    if ((rc = balloc(b, &d_inst, count)) || (rc = balloc(b, &d_order, count)) || (rc = balloc(b, &d_counter, 1)) ||
        (rc = balloc(b, &arp, rpa)) || (rc = balloc(b, &trp, rpt)) || (rc = balloc(b, &aci, nz)) ||
        (rc = balloc(b, &tci, nz)) || (rc = balloc(b, &av, nz)) || (rc = balloc(b, &tv, nz)) ||
        (rc = balloc(b, &oc, no)) || (rc = balloc(b, &olv, no)) || (rc = balloc(b, &ouv, no)) ||
        (rc = balloc(b, &olc, mo)) || (rc = balloc(b, &ouc, mo)))
        return bail(rc, "sp_batch_create: out of device memory");
    cudaStream_t st = ctx->stream;
    auto up = [&](void *d, const void *h, size_t bytes) -> int {
        if (bytes) SP_CUDA_TRY(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st));
        return SP_OK;
    };
    if ((rc = up(d_inst, b->inst.data(), sizeof(BatchInst) * count)) ||
        (rc = up(d_order, order.data(), sizeof(int) * count)) || (rc = up(arp, h_arp.data(), sizeof(int) * rpa)) ||
        (rc = up(trp, h_trp.data(), sizeof(int) * rpt)) || (rc = up(aci, h_aci.data(), sizeof(int) * nz)) ||
        (rc = up(tci, h_tci.data(), sizeof(int) * nz)) || (rc = up(av, h_av.data(), sizeof(double) * nz)) ||
        (rc = up(tv, h_tv.data(), sizeof(double) * nz)) || (rc = up(oc, h_c.data(), sizeof(double) * no)) ||
        (rc = up(olv, h_lv.data(), sizeof(double) * no)) || (rc = up(ouv, h_uv.data(), sizeof(double) * no)) ||
        (rc = up(olc, h_lc.data(), sizeof(double) * mo)) || (rc = up(ouc, h_uc.data(), sizeof(double) * mo)))
        return bail(rc, "sp_batch_create: upload failed");
    // The kernel scales the values in place, so every solve restarts from the originals.
    double *av0, *tv0;
    if ((rc = balloc(b, &av0, nz)) || (rc = balloc(b, &tv0, nz))) return bail(rc, "out of device memory");
    cudaMemcpyAsync(av0, av, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(tv0, tv, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st);
    A.inst = d_inst;
    A.order = d_order;
    A.counter = d_counter;
    A.a_rp = arp;
    A.a_ci = aci;
    A.t_rp = trp;
    A.t_ci = tci;
    A.a_v = av;
    A.t_v = tv;
    A.oc = oc;
    A.olv = olv;
    A.ouv = ouv;
    A.olc = olc;
    A.ouc = ouc;
    double **nvecs[] = {&A.c, &A.lv, &A.uv, &A.df, &A.cs, &A.x, &A.xt, &A.xbar, &A.xa, &A.aty, &A.pv, &A.ox};
    double **mvecs[] = {&A.lc, &A.uc, &A.pf, &A.rs, &A.y, &A.yt, &A.ya, &A.pt, &A.oy};
    for (double **p : nvecs)
        if ((rc = balloc(b, p, no))) return bail(rc, "out of device memory");
    for (double **p : mvecs)
        if ((rc = balloc(b, p, mo))) return bail(rc, "out of device memory");
    if ((rc = balloc(b, &A.pk, no)) || (rc = balloc(b, &A.pky, mo))) return bail(rc, "out of device memory");
    A.a_v32 = A.t_v32 = nullptr;
    A.xbar32 = A.y32 = nullptr;
    if (b->mixed) {
        if ((rc = balloc(b, &A.a_v32, nz)) || (rc = balloc(b, &A.t_v32, nz)) || (rc = balloc(b, &A.xbar32, no)) ||
            (rc = balloc(b, &A.y32, mo)))
            return bail(rc, "out of device memory");
    }
    if ((rc = balloc(b, &A.res, count))) return bail(rc, "out of device memory");
    if ((rc = balloc(b, &A.drain_ns, 1))) return bail(rc, "out of device memory");
    {
        double handoff_s = 2.0;
        if (const char *env = getenv("SP_BATCH_HANDOFF_S")) handoff_s = atof(env);
        A.handoff_ns = handoff_s > 0 ? (unsigned long long)(handoff_s * 1e9) : 0ull;
    }
    DevParams dp{};
    dp.tolerance = P.tolerance;
    dp.infeasibility_tolerance = P.infeasibility_tolerance;
    dp.max_iterations = P.max_iterations;
    dp.check_every = P.check_every;
    dp.reflection = P.reflection;
    dp.restart_sufficient = P.restart_sufficient;
    dp.restart_necessary = P.restart_necessary;
    dp.restart_artificial = P.restart_artificial;
    dp.pid_kp = P.pid_kp;
    dp.pid_ki = P.pid_ki;
    dp.pid_kd = P.pid_kd;
    dp.pid_discount = P.pid_discount;
    dp.termination = P.termination;
    dp.mixed = b->mixed;
    dp.mixed_switch_tolerance = P.mixed_switch_tolerance;
    dp.mixed_stall_checks = MIXED_STALL_CHECKS;
    dp.bound_objective_rescaling = P.bound_objective_rescaling;
    A.base = dp;
    A.power_iterations = P.power_iterations;
    A.geo_passes = P.geometric_mean_passes;
    A.ruiz_iterations = P.ruiz_iterations;
    A.pc_enabled = P.pock_chambolle_enabled;
    A.pc_alpha = P.pock_chambolle_alpha;
    A.rescale = P.bound_objective_rescaling;
    A.step_size_factor = P.step_size_factor;
    Tile *d_ta, *d_tt;
    if ((rc = balloc(b, &d_ta, n_ta)) || (rc = balloc(b, &d_tt, n_tt)) || (rc = balloc(b, &A.part, n_part)) ||
        (rc = up(d_ta, h_ta.data(), sizeof(Tile) * n_ta)) || (rc = up(d_tt, h_tt.data(), sizeof(Tile) * n_tt)))
        return bail(rc, "sp_batch_create: tile plans");
    A.a_tiles = d_ta;
    A.t_tiles = d_tt;
    const size_t smem = batch_smem_bytes();
    SP_CUDA_TRY(cudaFuncSetAttribute((const void *)k_batch<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<NT>, NT, smem));
    b->grid = std::max(1, std::min(count, std::max(1, per_sm) * ctx->sms));
    b->d_inst = d_inst;
    b->d_counter = d_counter;
    b->av0 = av0;
    b->tv0 = tv0;
    b->smem = smem;
    if (tune && (rc = tune_variants(b))) return bail(rc, "sp_batch_create: tuner");
    // one graph: restore the original values, reset the counter, run the persistent kernel
    cudaGraph_t g;
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    SP_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(av, av0, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(tv, tv0, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(d_counter, 0, sizeof(int), st);
    cudaMemsetAsync(A.drain_ns, 0, sizeof(unsigned long long), st);
    k_batch<NT><<<b->grid, NT, smem, st>>>(A);
    SP_CUDA_TRY(cudaStreamEndCapture(st, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bail(SP_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
    *out = b;
    return SP_OK;
}

}  // namespace sp

extern "C" int sp_batch_solve(sp_batch *b, sp_batch_result *results, double *elapsed_s) {
    if (!b) return SP_ERR_INVALID;
    int rc = enter(b->ctx);
    if (rc) return rc;
    cudaStream_t st = b->ctx->stream;
    EventPair ep;
    if ((rc = ep.init())) return rc;
    SP_CUDA_TRY(cudaEventRecord(ep.e0, st));
    SP_CUDA_TRY(cudaGraphLaunch(b->graph, st));
    SP_CUDA_TRY(cudaEventRecord(ep.e1, st));
    SP_CUDA_TRY(cudaEventSynchronize(ep.e1));
    float ms = 0.f;
    SP_CUDA_TRY(cudaEventElapsedTime(&ms, ep.e0, ep.e1));
    std::vector<sp_batch_result> res(b->count);
    SP_CUDA_TRY(cudaMemcpy(res.data(), b->args.res, sizeof(sp_batch_result) * b->count, cudaMemcpyDeviceToHost));
    const auto t0 = std::chrono::steady_clock::now();
    if ((rc = hand_off(b, res))) return rc;
    const double handoff_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (elapsed_s) *elapsed_s = ms * 1e-3 + handoff_s;
    if (results) std::copy(res.begin(), res.end(), results);
    return SP_OK;
}

extern "C" int sp_batch_download(sp_batch *b, int i, double *x, double *y) {
    if (!b || i < 0 || i >= b->count) return SP_ERR_INVALID;
    int rc = enter(b->ctx);
    if (rc) return rc;
    const BatchInst &I = b->inst[i];
    if (x && I.n) SP_CUDA_TRY(cudaMemcpy(x, b->args.ox + I.no, sizeof(double) * I.n, cudaMemcpyDeviceToHost));
    if (y && I.m) SP_CUDA_TRY(cudaMemcpy(y, b->args.oy + I.mo, sizeof(double) * I.m, cudaMemcpyDeviceToHost));
    return SP_OK;
}
