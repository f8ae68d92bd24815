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
#include <chrono>
#include <cstring>
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
};

namespace sp {

// Lanes per row for a matrix whose rows hold `mean` entries on average: the
// smallest power of two that leaves each lane about three products (one lane per
// row keeps the reference's summation order for short rows).
int lanes_for(double mean) {
    int L = 1;
    while (L < 32 && L * 3 < mean) L <<= 1;
    return L;
}

template <class T>
int balloc(sp_batch *b, T **p, int64_t n) {
    SP_CUDA_TRY(cudaMalloc(p, sizeof(T) * std::max<int64_t>(n, 1)));
    b->bufs.push_back(*p);
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
    if (!lps || count <= 0 || !out) return fail(SP_ERR_INVALID, "sp_batch_create: bad arguments");
    sp_solver_params P;
    sp_solver_params_default(&P);
    if (params) P = *params;
    auto *b = new sp_batch();
    b->ctx = ctx;
    b->count = count;
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
        I.lanes_a = lanes_for(A.nrows ? (double)A.nnz / A.nrows : 0.0);
        I.lanes_t = lanes_for(A.ncols ? (double)A.nnz / A.ncols : 0.0);
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
    A.a_v32 = A.t_v32 = nullptr;
    A.xbar32 = A.y32 = nullptr;
    if (b->mixed) {
        if ((rc = balloc(b, &A.a_v32, nz)) || (rc = balloc(b, &A.t_v32, nz)) || (rc = balloc(b, &A.xbar32, no)) ||
            (rc = balloc(b, &A.y32, mo)))
            return bail(rc, "out of device memory");
    }
    if ((rc = balloc(b, &A.res, count))) return bail(rc, "out of device memory");
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
    dp.bound_objective_rescaling = P.bound_objective_rescaling;
    A.base = dp;
    A.power_iterations = P.power_iterations;
    A.geo_passes = P.geometric_mean_passes;
    A.ruiz_iterations = P.ruiz_iterations;
    A.pc_enabled = P.pock_chambolle_enabled;
    A.pc_alpha = P.pock_chambolle_alpha;
    A.rescale = P.bound_objective_rescaling;
    A.step_size_factor = P.step_size_factor;
    // one graph: restore the original values, reset the counter, run the persistent kernel
    int per_sm = 0;
    SP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<NT>, NT, 0));
    b->grid = std::max(1, std::min(count, std::max(1, per_sm) * ctx->sms));
    cudaGraph_t g;
    SP_CUDA_TRY(cudaStreamSynchronize(st));
    SP_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(av, av0, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(tv, tv0, sizeof(double) * nz, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(d_counter, 0, sizeof(int), st);
    k_batch<NT><<<b->grid, NT, 0, st>>>(A);
    SP_CUDA_TRY(cudaStreamEndCapture(st, &g));
    cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bail(SP_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
    *out = b;
    return SP_OK;
}

extern "C" int sp_batch_solve(sp_batch *b, sp_batch_result *results, double *elapsed_s) {
    if (!b) return SP_ERR_INVALID;
    int rc = enter(b->ctx);
    if (rc) return rc;
    cudaStream_t st = b->ctx->stream;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    SP_CUDA_TRY(cudaGraphLaunch(b->graph, st));
    cudaEventRecord(e1, st);
    SP_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (elapsed_s) *elapsed_s = ms * 1e-3;
    if (results)
        SP_CUDA_TRY(cudaMemcpy(results, b->args.res, sizeof(sp_batch_result) * b->count, cudaMemcpyDeviceToHost));
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
