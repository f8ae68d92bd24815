// serve.cu — the serving loop (Part 4 of the C ABI): continuous batching of
// arriving LPs on one GPU under an HBM budget.
//
// Requests are copied on submit and queued. Admission is first come, first served
// by HBM footprint (sp_server_footprint): a request is admitted when its
// footprint fits in what the budget has left. Admitted requests run
//   * on one of `max_inflight` solve slots when larger than `batch_max_nnz`: each
//     slot is a host thread with its own context (own CUDA stream) running the
//     device-resident solve, so the epochs of different requests overlap on the
//     GPU and a slot takes the next request as soon as its solve ends;
//   * otherwise in the next launch of the batched persistent kernel, which the
//     batching thread assembles from every small request waiting when the previous
//     launch ends.
// A request's kernels never read another request's memory and each solve is
// deterministic, so a result is the same alone and in any mix.
#include <algorithm>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "control.cuh"
#include "internal.cuh"

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    int64_t id = 0;
    int64_t footprint = 0;
    bool small = false;
    // owned copy of the LP
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v, c, lc, uc, lv, uv;
    double c0 = 0;
    int maximize = 0;
    sp_lp lp{};
    // timing and result
    double t_submit = 0, t_admit = 0, t_done = 0;
    sp_server_result res{};
    std::vector<double> x, y;
    int error = SP_OK;

    void bind() {
        lp.a.nrows = (int64_t)rp.size() - 1;
        lp.a.ncols = (int64_t)c.size();
        lp.a.nnz = (int64_t)v.size();
        lp.a.row_ptr = rp.data();
        lp.a.col_idx = ci.data();
        lp.a.values = v.data();
        lp.c = c.data();
        lp.lc = lc.data();
        lp.uc = uc.data();
        lp.lv = lv.data();
        lp.uv = uv.data();
        lp.c0 = c0;
        lp.maximize = maximize;
    }
};

}  // namespace

struct sp_server {
    sp_ctx *ctx = nullptr;
    sp_server_config cfg{};
    sp_solver_params params{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;   // submitted, not admitted
    std::deque<Request *> small_q;   // admitted small requests waiting for the next batch
    std::deque<Request *> finished;  // results not yet polled
    double budget_used = 0;
    bool stop = false;
    int64_t next_id = 1;
    std::vector<std::thread> workers;
    std::vector<sp_ctx *> slot_ctx;
    sp_ctx *batch_ctx = nullptr;
    std::thread batcher;

    // Admits from the head of the queue while the budget allows; returns a large
    // request for the calling slot, or null. Small ones move to the batch queue.
    Request *admit_locked(bool want_large) {
        while (!pending.empty()) {
            Request *r = pending.front();
            if (budget_used + (double)r->footprint > cfg.budget_bytes && budget_used > 0) return nullptr;
            if (!r->small && !want_large) return nullptr;
            pending.pop_front();
            budget_used += (double)r->footprint;
            r->t_admit = now_s();
            if (r->small) {
                small_q.push_back(r);
                cv_work.notify_all();
                continue;
            }
            return r;
        }
        return nullptr;
    }

    void finish(Request *r) {
        std::lock_guard<std::mutex> lock(mu);
        r->t_done = now_s();
        budget_used -= (double)r->footprint;
        r->res.queue_s = r->t_admit - r->t_submit;
        r->res.solve_s = r->t_done - r->t_admit;
        r->res.total_s = r->t_done - r->t_submit;
        finished.push_back(r);
        cv_done.notify_all();
        cv_work.notify_all();
    }

    void slot_loop(int slot) {
        sp_ctx *ctx = slot_ctx[slot];
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait(lock, [&] {
                    if (stop) return true;
                    r = admit_locked(true);
                    return r != nullptr;
                });
                if (!r) return;  // stopping
            }
            sp_solution_info info{};
            r->x.assign(r->lp.a.ncols, 0.0);
            r->y.assign(r->lp.a.nrows, 0.0);
            r->error = sp_solve(ctx, &r->lp, &params, r->x.data(), r->y.data(), &info);
            r->res.status = r->error ? -1 : info.status;
            r->res.error = r->error;
            r->res.path = 0;
            if (r->error) snprintf(r->res.message, sizeof r->res.message, "%s", sp_ctx_last_error(ctx));
            r->res.objective = info.objective;
            r->res.dual_objective = info.dual_objective;
            r->res.primal_residual = info.primal_residual;
            r->res.dual_residual = info.dual_residual;
            r->res.gap = info.gap;
            r->res.iterations = info.iterations;
            finish(r);
        }
    }

    void batch_loop() {
        for (;;) {
            std::vector<Request *> group;
            {
                std::unique_lock<std::mutex> lock(mu);
                cv_work.wait(lock, [&] {
                    admit_locked(false);
                    return stop || !small_q.empty();
                });
                if (stop && small_q.empty()) return;
                group.assign(small_q.begin(), small_q.end());
                small_q.clear();
            }
            std::vector<sp_lp> lps;
            for (Request *r : group) lps.push_back(r->lp);
            sp_batch *b = nullptr;
            std::vector<sp_batch_result> res(group.size());
            int rc = sp_batch_create(batch_ctx, lps.data(), (int)lps.size(), &params, &b);
            if (!rc) rc = sp_batch_solve(b, res.data(), nullptr);
            for (size_t i = 0; i < group.size(); ++i) {
                Request *r = group[i];
                r->x.assign(r->lp.a.ncols, 0.0);
                r->y.assign(r->lp.a.nrows, 0.0);
                if (!rc) rc = sp_batch_download(b, (int)i, r->x.data(), r->y.data());
                r->error = rc;
                r->res.status = rc ? -1 : res[i].status;
                r->res.error = rc;
                r->res.path = 1;
                if (rc) snprintf(r->res.message, sizeof r->res.message, "%s", sp_ctx_last_error(batch_ctx));
                r->res.objective = res[i].objective;
                r->res.dual_objective = res[i].dual_objective;
                r->res.primal_residual = res[i].primal_residual;
                r->res.dual_residual = res[i].dual_residual;
                r->res.gap = res[i].gap;
                r->res.iterations = res[i].iterations;
            }
            sp_batch_free(b);
            for (Request *r : group) finish(r);
        }
    }
};

extern "C" int64_t sp_server_footprint(int64_t m, int64_t n, int64_t nnz, int precision) {
    // A' and A'ᵀ (int32 index + FP64 value), their FP32 copies in the mixed form,
    // the transpose's sort buffers at set-up (about 24 bytes per nonzero), the SELL
    // copy of A' (at most two slots per nonzero, 12 or 16 bytes each, and at most 18 bytes
    // per row for its lengths, order, warp-row list, chunk and slice offsets, the last
    // window padded, plus the check's 64 bytes of row contributions), the n- and m-vectors
    // of the solve, and 8 MiB of fixed overhead.
    int64_t b = 2 * nnz * 12 + 24 * nnz + 4 * (m + n + 2);
    if (precision == SP_PRECISION_MIXED) b += 2 * nnz * 4 + 4 * (m + n);
    b += 2 * nnz * (precision == SP_PRECISION_MIXED ? 16 : 12) + (18 + 8 * sp::NP_D) * (m + 1024) + 2 * 1024 * 16;
    b += 168 * n + 120 * m + (8ll << 20);
    return b;
}

extern "C" int sp_server_create(sp_ctx *ctx, const sp_server_config *cfg, const sp_solver_params *params,
                                sp_server **out) {
    if (!ctx || !cfg || !out || cfg->max_inflight < 1) return SP_ERR_INVALID;
    auto *s = new sp_server();
    s->ctx = ctx;
    s->cfg = *cfg;
    sp_solver_params_default(&s->params);
    if (params) s->params = *params;
    for (int i = 0; i < cfg->max_inflight; ++i) {
        sp_ctx *c = nullptr;
        int rc = sp_ctx_create(ctx->device, &c);
        if (rc) {
            sp_server_destroy(s);
            return rc;
        }
        s->slot_ctx.push_back(c);
    }
    int rc = sp_ctx_create(ctx->device, &s->batch_ctx);
    if (rc) {
        sp_server_destroy(s);
        return rc;
    }
    for (int i = 0; i < cfg->max_inflight; ++i) s->workers.emplace_back(&sp_server::slot_loop, s, i);
    s->batcher = std::thread(&sp_server::batch_loop, s);
    *out = s;
    return SP_OK;
}

extern "C" int sp_server_submit(sp_server *s, const sp_lp *lp, int64_t *id) {
    if (!s || !lp || !lp->a.row_ptr) return SP_ERR_INVALID;
    // an invalid LP is turned away here, before it can share a batch with valid ones
    char msg[256] = "";
    const int v = sp_problem_validate(lp, msg, sizeof msg);
    if (v != SP_OK) {
        if (sp::enter(s->ctx) == SP_OK) sp::fail(v, msg);
        return v;
    }
    auto *r = new Request();
    const int64_t m = lp->a.nrows, n = lp->a.ncols, nnz = lp->a.nnz;
    r->rp.assign(lp->a.row_ptr, lp->a.row_ptr + m + 1);
    r->ci.assign(lp->a.col_idx, lp->a.col_idx + nnz);
    r->v.assign(lp->a.values, lp->a.values + nnz);
    r->c.assign(lp->c, lp->c + n);
    r->lv.assign(lp->lv, lp->lv + n);
    r->uv.assign(lp->uv, lp->uv + n);
    r->lc.assign(lp->lc, lp->lc + m);
    r->uc.assign(lp->uc, lp->uc + m);
    r->c0 = lp->c0;
    r->maximize = lp->maximize;
    r->bind();
    r->footprint = sp_server_footprint(m, n, nnz, s->params.precision);
    r->small = nnz <= s->cfg.batch_max_nnz;
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->next_id++;
    r->res.id = r->id;
    r->res.footprint_bytes = r->footprint;
    r->t_submit = now_s();
    s->pending.push_back(r);
    if (id) *id = r->id;
    s->cv_work.notify_all();
    return SP_OK;
}

extern "C" int sp_server_poll(sp_server *s, double timeout_s, sp_server_result *out, double *x, int64_t xcap,
                              double *y, int64_t ycap, int *got) {
    if (!s || !out || !got) return SP_ERR_INVALID;
    *got = 0;
    Request *r = nullptr;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        auto ready = [&] { return !s->finished.empty(); };
        if (timeout_s < 0) s->cv_done.wait(lock, ready);
        else s->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready);
        if (s->finished.empty()) return SP_OK;
        r = s->finished.front();
        // a solution buffer too small for this result: leave the result queued so the
        // caller can poll again with larger buffers
        if ((x && xcap < (int64_t)r->x.size()) || (y && ycap < (int64_t)r->y.size())) return SP_ERR_INVALID;
        s->finished.pop_front();
    }
    *out = r->res;
    if (x) memcpy(x, r->x.data(), sizeof(double) * r->x.size());
    if (y) memcpy(y, r->y.data(), sizeof(double) * r->y.size());
    int err = r->error;
    delete r;
    *got = 1;
    return err;
}

extern "C" void sp_server_destroy(sp_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers)
        if (t.joinable()) t.join();
    if (s->batcher.joinable()) s->batcher.join();
    for (Request *r : s->pending) delete r;
    for (Request *r : s->small_q) delete r;
    for (Request *r : s->finished) delete r;
    for (sp_ctx *c : s->slot_ctx) sp_ctx_destroy(c);
    sp_ctx_destroy(s->batch_ctx);
    delete s;
}
