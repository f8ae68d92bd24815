// backend.cu — the Backend trait (crates/saddlepoint-core/src/backend.rs:43-137)
// as C entry points on one CUDA stream: context, vectors, problem load, the
// element-wise steps, the SpMVs and the reductions.
//
// The reference GPU backend (crates/saddlepoint-cuda/src/backend.rs) uses
// cuSPARSE for SpMV and sums per-block partials on the host. Here the SpMV is the
// row-tile kernel of tiles.cuh and every reduction finishes on the device in a
// fixed order (a second one-block pass), so only the final scalars cross to the
// host and results are identical from run to run.
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.cuh"
#include "tiles.cuh"

namespace sp {

static thread_local sp_ctx *t_ctx = nullptr;
void set_current_ctx(sp_ctx *ctx) { t_ctx = ctx; }
int fail(int code, const std::string &msg) {
    if (t_ctx) t_ctx->last_error = msg;
    return code;
}

// ---------------------------------------------------------------- kernels

struct StoreOp {  // out = A x (Backend::spmv / spmv_t)
    using VT = double;
    using ST = double;
    static constexpr int G = 1, NP = 0;
    static constexpr unsigned F32 = 0;
    const int *rp, *ci;
    const double *vals;
    const Tile *tiles;
    const double *x;
    double *out;
    const uint16_t *sched;
    struct Pre {};
    __device__ bool setup() { return true; }
    __device__ __forceinline__ Pre pre(int) const { return {}; }
    __device__ __forceinline__ void prod(int c, double v, double (&p)[1]) const { p[0] = v * __ldg(x + c); }
    __device__ __forceinline__ void row(int r, const double (&s)[1], double *, const Pre &) const { out[r] = s[0]; }
    __device__ void store(int, const double *) const {}
};

#define GRID_LOOP(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

__global__ void k_primal_step(const double *__restrict__ x, const double *__restrict__ aty,
                              const double *__restrict__ c, const double *__restrict__ lv,
                              const double *__restrict__ uv, double tau, double *__restrict__ x_t,
                              double *__restrict__ x_bar, int64_t n) {
    GRID_LOOP(j, n) {  // cpu lib.rs:156-158
        const double xj = x[j];
        const double t = clampd(xj - tau * (c[j] - aty[j]), lv[j], uv[j]);
        x_t[j] = t;
        x_bar[j] = 2.0 * t - xj;
    }
}

__global__ void k_dual_step(const double *__restrict__ y, const double *__restrict__ ax,
                            const double *__restrict__ lc, const double *__restrict__ uc, double sigma,
                            double *__restrict__ y_t, int64_t m) {
    GRID_LOOP(i, m) {  // cpu lib.rs:170-173
        const double a = ax[i], yi = y[i];
        const double v = a - yi / sigma;
        y_t[i] = yi - sigma * (a - clampd(v, lc[i], uc[i]));
    }
}

__global__ void k_halpern(double *__restrict__ z, const double *__restrict__ zt, const double *__restrict__ an,
                          double w, double rho, int64_t n) {
    GRID_LOOP(i, n) { z[i] = halpern(z[i], zt[i], an[i], w, rho); }
}

__global__ void k_sub(const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ o, int64_t n) {
    GRID_LOOP(i, n) { o[i] = a[i] - b[i]; }
}

__global__ void k_scale(double *__restrict__ v, double alpha, int64_t n) {
    GRID_LOOP(i, n) { v[i] *= alpha; }
}

// Stage one of a reduction: K sums of F(i) over a grid-stride slice per block.
template <int K, class F>
__global__ void __launch_bounds__(NT) k_reduce(F f, int64_t n, double *__restrict__ partials) {
    __shared__ double sh[K * (NT / 32)];
    double s[K];
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] = 0.0;
    GRID_LOOP(i, n) { f(i, s); }
    block_sum<K>(s, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) partials[blockIdx.x * K + k] = s[k];
    }
}

struct RedRegion {
    int offset, blocks, k;
};
struct RedPlan {
    RedRegion r[4];
    int n;
};

// Stage two: one block adds the per-block partials of every region in block order.
__global__ void __launch_bounds__(NT) k_reduce_final(const double *__restrict__ partials, RedPlan plan,
                                                    double *__restrict__ out) {
    __shared__ double sh[NT / 32];
    int slot = 0;
    for (int g = 0; g < plan.n; ++g) {
        const RedRegion r = plan.r[g];
        for (int k = 0; k < r.k; ++k) {
            double s[1] = {0.0};
            for (int b = threadIdx.x; b < r.blocks; b += NT) s[0] += partials[r.offset + b * r.k + k];
            block_sum<1>(s, sh);
            if (threadIdx.x == 0) out[slot] = s[0];
            ++slot;
        }
    }
}

// Element functors of the reductions (crates/saddlepoint-cpu/src/lib.rs:189-259).
struct FDist {
    const double *a, *b;
    __device__ void operator()(int64_t i, double (&s)[1]) const { double d = a[i] - b[i]; s[0] += d * d; }
};
struct FDot {
    const double *a, *b;
    __device__ void operator()(int64_t i, double (&s)[1]) const { s[0] += a[i] * b[i]; }
};
struct FPrimRes {
    const double *ax, *lc, *uc, *pf;
    __device__ void operator()(int64_t i, double (&s)[1]) const {
        double e = excess(ax[i], lc[i], uc[i]) * pf[i];
        s[0] += e * e;
    }
};
struct FDualRows {
    const double *y, *lc, *uc;
    __device__ void operator()(int64_t i, double (&s)[1]) const { s[0] += bound_term(y[i], lc[i], uc[i]); }
};
struct FDualCols {
    const double *c, *aty, *lv, *uv, *df;
    __device__ void operator()(int64_t j, double (&s)[2]) const {
        double r = c[j] - aty[j];
        double f = forbidden(r, lv[j], uv[j]) * df[j];
        s[0] += f * f;
        s[1] += bound_term(r, lv[j], uv[j]);
    }
};
struct FStepDual {
    const double *x, *xt, *aty, *atyt, *df;
    double inv_tau;
    __device__ void operator()(int64_t j, double (&s)[1]) const {
        double r = (aty[j] - atyt[j] - (xt[j] - x[j]) * inv_tau) * df[j];
        s[0] += r * r;
    }
};
struct FPRayRows {
    const double *adx, *lc, *uc;
    __device__ void operator()(int64_t i, double (&s)[1]) const {
        double v = recession_violation(adx[i], lc[i], uc[i]);
        s[0] += v * v;
    }
};
struct FPRayCols {
    const double *dx, *c, *lv, *uv;
    __device__ void operator()(int64_t j, double (&s)[3]) const {
        double d = dx[j], v = recession_violation(d, lv[j], uv[j]);
        s[0] += v * v;
        s[1] += d * d;
        s[2] += c[j] * d;
    }
};
struct FDRayRows {
    const double *dy, *lc, *uc;
    __device__ void operator()(int64_t i, double (&s)[3]) const {
        double d = dy[i], f = forbidden(d, lc[i], uc[i]);
        s[0] += f * f;
        s[1] += bound_term(d, lc[i], uc[i]);
        s[2] += d * d;
    }
};
struct FDRayCols {
    const double *atdy, *lv, *uv;
    __device__ void operator()(int64_t j, double (&s)[2]) const {
        double r = -atdy[j], f = forbidden(r, lv[j], uv[j]);
        s[0] += f * f;
        s[1] += bound_term(r, lv[j], uv[j]);
    }
};

// ---------------------------------------------------------------- helpers

static int grid_for(const sp_ctx *ctx, int64_t n) {
    int64_t b = (n + NT - 1) / NT;
    int64_t cap = (int64_t)ctx->sms * 32;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

// A reduction call: queue stage-one kernels, then finish and read back once.
struct Reduction {
    sp_ctx *ctx;
    RedPlan plan{};
    int offset = 0, slots = 0;
    explicit Reduction(sp_ctx *c) : ctx(c) {}
    template <int K, class F>
    void add(F f, int64_t n) {
        int blocks = (int)std::min<int64_t>(RED_BLOCKS, std::max<int64_t>(1, (n + NT - 1) / NT));
        k_reduce<K><<<blocks, NT, 0, ctx->stream>>>(f, n, ctx->d_partials + offset);
        plan.r[plan.n++] = RedRegion{offset, blocks, K};
        offset += blocks * K;
        slots += K;
    }
    int finish(double *out) {
        k_reduce_final<<<1, NT, 0, ctx->stream>>>(ctx->d_partials, plan, ctx->d_result);
        SP_CUDA_TRY(cudaGetLastError());
        SP_CUDA_TRY(cudaMemcpyAsync(ctx->h_result, ctx->d_result, sizeof(double) * slots, cudaMemcpyDeviceToHost,
                                    ctx->stream));
        SP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        memcpy(out, ctx->h_result, sizeof(double) * slots);
        return SP_OK;
    }
};


}  // namespace sp

using namespace sp;

// ====================================================================== context

extern "C" int sp_ctx_create(int ordinal, sp_ctx **out) {
    if (!out) return SP_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= ordinal || ordinal < 0) {
        cudaGetLastError();
        return SP_ERR_UNAVAILABLE;
    }
    auto *ctx = new sp_ctx();
    set_current_ctx(ctx);
    ctx->device = ordinal;
    cudaDeviceProp prop;
    if (cudaSetDevice(ordinal) != cudaSuccess || cudaGetDeviceProperties(&prop, ordinal) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return SP_ERR_UNAVAILABLE;
    }
    ctx->sms = prop.multiProcessorCount;
    ctx->name = prop.name;
    keep_pool_memory(ordinal);
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->aux_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&ctx->d_partials, sizeof(double) * RED_BLOCKS * RED_SLOTS * 4) != cudaSuccess ||
        cudaMalloc(&ctx->d_result, sizeof(double) * RED_SLOTS * 4) != cudaSuccess ||
        cudaMallocHost(&ctx->h_result, sizeof(double) * RED_SLOTS * 4) != cudaSuccess ||
        cudaMalloc(&ctx->d_tiles, sizeof(int) * 2) != cudaSuccess ||
        cudaMemsetAsync(ctx->d_tiles, 0, sizeof(int) * 2, ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        sp_ctx_destroy(ctx);
        return SP_ERR_UNAVAILABLE;
    }
    *out = ctx;
    return SP_OK;
}

extern "C" void sp_ctx_destroy(sp_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->aux) cudaStreamSynchronize(ctx->aux);
    cudaFree(ctx->d_partials);
    cudaFree(ctx->d_result);
    cudaFreeHost(ctx->h_result);
    cudaFree(ctx->d_tiles);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->aux) cudaStreamDestroy(ctx->aux);
    if (ctx->aux_ev) cudaEventDestroy(ctx->aux_ev);
    if (t_ctx_is(ctx)) set_current_ctx(nullptr);
    delete ctx;
}

namespace sp {
bool t_ctx_is(const sp_ctx *c) { return t_ctx == c; }

// Device memory of problems and solvers comes from the device's stream-ordered pool,
// allocated and released on the context's stream. The pool keeps what is released
// (release threshold: unlimited), so a solve after a solve reuses mapped memory
// instead of paying cudaMalloc/cudaFree's mapping, unmapping and device-wide
// synchronisation again (0.1-1.2 s per 40M-nonzero solve, measured).
void keep_pool_memory(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    done[device] = true;
}

int dmalloc(void **p, size_t bytes) {
    cudaStream_t st = t_ctx ? t_ctx->stream : nullptr;
    cudaError_t e = cudaMallocAsync(p, std::max<size_t>(bytes, 16), st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(SP_ERR_CUDA, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    }
    return SP_OK;
}

void dfree(void *p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
}
int enter(sp_ctx *ctx) {
    if (!ctx) return SP_ERR_INVALID;
    set_current_ctx(ctx);
    ctx->last_error.clear();
    if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(SP_ERR_CUDA, "cudaSetDevice failed");
    return SP_OK;
}
}  // namespace sp

extern "C" const char *sp_ctx_last_error(const sp_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

extern "C" int sp_ctx_name(const sp_ctx *ctx, char *buf, size_t cap) {
    if (!ctx || !buf || cap == 0) return SP_ERR_INVALID;
    std::string n = "b200 (" + ctx->name + ")";
    snprintf(buf, cap, "%s", n.c_str());
    return SP_OK;
}

extern "C" void *sp_ctx_stream(sp_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// ====================================================================== vectors

extern "C" int sp_vec_upload(sp_ctx *ctx, const double *data, int64_t len, sp_vec **out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out || len < 0 || (len > 0 && !data)) return fail(SP_ERR_INVALID, "sp_vec_upload: bad arguments");
    auto *v = new sp_vec();
    v->ctx = ctx;
    v->n = len;
    if (cudaMalloc(&v->d, sizeof(double) * (len > 0 ? len : 1)) != cudaSuccess) {
        delete v;
        cudaGetLastError();
        return fail(SP_ERR_CUDA, "sp_vec_upload: out of device memory");
    }
    if (len > 0) {
        cudaError_t e = cudaMemcpyAsync(v->d, data, sizeof(double) * len, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            cudaFree(v->d);
            delete v;
            return fail(SP_ERR_CUDA, std::string("sp_vec_upload: ") + cudaGetErrorString(e));
        }
    }
    *out = v;
    return SP_OK;
}

extern "C" int sp_vec_download(sp_ctx *ctx, const sp_vec *v, double *out, int64_t len) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!v || len != v->n || (len > 0 && !out)) return fail(SP_ERR_INVALID, "sp_vec_download: length mismatch");
    if (len == 0) return SP_OK;
    SP_CUDA_TRY(cudaMemcpyAsync(out, v->d, sizeof(double) * len, cudaMemcpyDeviceToHost, ctx->stream));
    SP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return SP_OK;
}

extern "C" int sp_vec_copy(sp_ctx *ctx, const sp_vec *src, sp_vec *dst) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!src || !dst || src->n != dst->n) return fail(SP_ERR_INVALID, "sp_vec_copy: length mismatch");
    if (src->n == 0) return SP_OK;
    SP_CUDA_TRY(cudaMemcpyAsync(dst->d, src->d, sizeof(double) * src->n, cudaMemcpyDeviceToDevice, ctx->stream));
    return SP_OK;
}

extern "C" void sp_vec_free(sp_vec *v) {
    if (!v) return;
    cudaSetDevice(v->ctx->device);
    cudaStreamSynchronize(v->ctx->stream);
    cudaFree(v->d);
    delete v;
}

extern "C" int64_t sp_vec_len(const sp_vec *v) { return v ? v->n : -1; }

// ====================================================================== problem

namespace sp {

// Uploads one host CSR: int64 row pointers narrowed to int32 (TooLarge past 2^31-1,
// like CsrDevice::new in crates/saddlepoint-cuda/src/sparse.rs:52-91), the tile plan.
int upload_csr(sp_ctx *ctx, const sp_csr *h, DevCsr *d, bool want_f32) {
    if (!h || h->nrows < 0 || h->ncols < 0 || h->nnz < 0 || !h->row_ptr) return fail(SP_ERR_INVALID, "bad CSR");
    if (h->nnz > INT32_MAX - 1 || h->nrows > INT32_MAX - 1 || h->ncols > INT32_MAX - 1)
        return fail(SP_ERR_TOO_LARGE, "problem too large for 32-bit sparse indices");
    if (h->row_ptr[0] != 0 || h->row_ptr[h->nrows] != h->nnz) return fail(SP_ERR_INVALID, "CSR row_ptr inconsistent");
    d->nrows = h->nrows;
    d->ncols = h->ncols;
    d->nnz = h->nnz;
    std::vector<int> rp32(h->nrows + 1);
    for (int64_t i = 0; i <= h->nrows; ++i) {
        if (i > 0 && h->row_ptr[i] < h->row_ptr[i - 1]) return fail(SP_ERR_INVALID, "CSR row_ptr not monotone");
        rp32[i] = (int)h->row_ptr[i];
    }
    size_t nz = (size_t)std::max<int64_t>(h->nnz, 1) + CSR_PAD;
    int rc;
    if ((rc = dmalloc((void **)&d->rp, sizeof(int) * (h->nrows + 1 + CSR_PAD))) ||
        (rc = dmalloc((void **)&d->ci, sizeof(int) * nz)) || (rc = dmalloc((void **)&d->v, sizeof(double) * nz)))
        return rc;
    // the copies first: from page-locked memory they run while the host builds the tile plan
    SP_CUDA_TRY(cudaMemcpyAsync(d->rp, rp32.data(), sizeof(int) * (h->nrows + 1), cudaMemcpyHostToDevice, ctx->stream));
    if (h->nnz) {
        SP_CUDA_TRY(cudaMemcpyAsync(d->ci, h->col_idx, sizeof(int) * h->nnz, cudaMemcpyHostToDevice, ctx->stream));
        SP_CUDA_TRY(cudaMemcpyAsync(d->v, h->values, sizeof(double) * h->nnz, cudaMemcpyHostToDevice, ctx->stream));
    }
    // an early return waits for the copies, which read the caller's memory and rp32
    auto bail = [&](int code) {
        cudaStreamSynchronize(ctx->stream);
        return code;
    };
    std::vector<Tile> tiles = build_tiles(h->row_ptr, h->nrows);
    d->ntiles = (int)tiles.size();
    d->nlong = count_long_tiles(tiles);
    if ((rc = dmalloc((void **)&d->tiles, sizeof(Tile) * std::max<size_t>(tiles.size(), 1)))) return bail(rc);
    if (!tiles.empty())
        SP_CUDA_TRY(cudaMemcpyAsync(d->tiles, tiles.data(), sizeof(Tile) * tiles.size(), cudaMemcpyHostToDevice,
                                    ctx->stream));
    const std::vector<uint16_t> sched = build_schedule(h->row_ptr, h->nrows, tiles);
    if ((rc = dmalloc((void **)&d->sched, sizeof(uint16_t) * (std::max<int64_t>(h->nrows, 1) + CSR_PAD))))
        return bail(rc);
    if (h->nrows)
        SP_CUDA_TRY(cudaMemcpyAsync(d->sched, sched.data(), sizeof(uint16_t) * h->nrows, cudaMemcpyHostToDevice,
                                    ctx->stream));
    if (want_f32) {
        if ((rc = dmalloc((void **)&d->v32, sizeof(float) * nz))) return bail(rc);
    }
    // the host vectors die with this call
    SP_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return SP_OK;
}

void free_csr(DevCsr *d, cudaStream_t st) {
    for (void *p : {(void *)d->rp, (void *)d->ci, (void *)d->v, (void *)d->v32, (void *)d->tiles, (void *)d->sched})
        dfree(p, st);
    *d = DevCsr{};
}

int upload_vec(sp_ctx *ctx, double **d, const double *h, int64_t n) {
    int rc = dmalloc((void **)d, sizeof(double) * (std::max<int64_t>(n, 1) + CSR_PAD));
    if (rc) return rc;
    if (n) SP_CUDA_TRY(cudaMemcpyAsync(*d, h, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    return SP_OK;
}

void launch_spmv(sp_ctx *ctx, const DevCsr &A, const double *x, double *out, cudaStream_t s) {
    if (A.ntiles == 0) return;
    StoreOp op{A.rp, A.ci, A.v, A.tiles, x, out, A.sched};
    k_tiles<StoreOp><<<A.ntiles, NT, tile_smem_bytes<1, double>(), s>>>(op);
}

}  // namespace sp

extern "C" int sp_problem_load(sp_ctx *ctx, const sp_csr *a, const sp_csr *at, const double *c, const double *lc,
                               const double *uc, const double *lv, const double *uv, const double *primal_factor,
                               const double *dual_factor, sp_problem **out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!a || !at || !out || !c || !lc || !uc || !lv || !uv || !primal_factor || !dual_factor)
        return fail(SP_ERR_INVALID, "sp_problem_load: null argument");
    if (at->nrows != a->ncols || at->ncols != a->nrows || at->nnz != a->nnz)
        return fail(SP_ERR_INVALID, "sp_problem_load: `at` is not the transpose's shape");
    // a column index out of range would make the SpMV read outside its vector on the GPU
    auto cols_ok = [](const sp_csr *M) {
        if (M->nnz > 0 && !M->col_idx) return false;
        for (int64_t k = 0; k < M->nnz; ++k)
            if (M->col_idx[k] < 0 || M->col_idx[k] >= M->ncols) return false;
        return true;
    };
    if (!cols_ok(a) || !cols_ok(at)) return fail(SP_ERR_INVALID, "sp_problem_load: a column index is out of range");
    auto *p = new sp_problem();
    p->ctx = ctx;
    p->m = a->nrows;
    p->n = a->ncols;
    int64_t m = p->m, n = p->n;
    if ((rc = upload_csr(ctx, a, &p->a, false)) || (rc = upload_csr(ctx, at, &p->at, false)) ||
        (rc = upload_vec(ctx, &p->c, c, n)) || (rc = upload_vec(ctx, &p->lc, lc, m)) ||
        (rc = upload_vec(ctx, &p->uc, uc, m)) || (rc = upload_vec(ctx, &p->lv, lv, n)) ||
        (rc = upload_vec(ctx, &p->uv, uv, n)) || (rc = upload_vec(ctx, &p->pf, primal_factor, m)) ||
        (rc = upload_vec(ctx, &p->df, dual_factor, n))) {
        sp_problem_free(p);
        return rc;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        sp_problem_free(p);
        return fail(SP_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = p;
    return SP_OK;
}

extern "C" void sp_problem_free(sp_problem *p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    free_csr(&p->a, p->ctx->stream);
    free_csr(&p->at, p->ctx->stream);
    for (double *v : {p->c, p->lc, p->uc, p->lv, p->uv, p->pf, p->df}) dfree(v, p->ctx->stream);
    cudaStreamSynchronize(p->ctx->stream);
    delete p;
}

// ====================================================================== trait methods

#define CHECK_LEN(v, len, what) \
    if (!(v) || (v)->n != (len)) return fail(SP_ERR_INVALID, std::string(what) + ": vector length mismatch")

extern "C" int sp_spmv(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, sp_vec *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p) return fail(SP_ERR_INVALID, "sp_spmv: null problem");
    CHECK_LEN(x, p->n, "sp_spmv x");
    CHECK_LEN(out, p->m, "sp_spmv out");
    launch_spmv(ctx, p->a, x->d, out->d, ctx->stream);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_spmv_t(sp_ctx *ctx, const sp_problem *p, const sp_vec *y, sp_vec *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p) return fail(SP_ERR_INVALID, "sp_spmv_t: null problem");
    CHECK_LEN(y, p->m, "sp_spmv_t y");
    CHECK_LEN(out, p->n, "sp_spmv_t out");
    launch_spmv(ctx, p->at, y->d, out->d, ctx->stream);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_primal_step(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, const sp_vec *aty, double tau,
                              sp_vec *x_t, sp_vec *x_bar) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p) return fail(SP_ERR_INVALID, "sp_primal_step: null problem");
    int64_t n = p->n;
    CHECK_LEN(x, n, "sp_primal_step x");
    CHECK_LEN(aty, n, "sp_primal_step aty");
    CHECK_LEN(x_t, n, "sp_primal_step x_t");
    CHECK_LEN(x_bar, n, "sp_primal_step x_bar");
    if (n == 0) return SP_OK;
    k_primal_step<<<grid_for(ctx, n), NT, 0, ctx->stream>>>(x->d, aty->d, p->c, p->lv, p->uv, tau, x_t->d, x_bar->d, n);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_dual_step(sp_ctx *ctx, const sp_problem *p, const sp_vec *y, const sp_vec *ax_bar, double sigma,
                            sp_vec *y_t) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p) return fail(SP_ERR_INVALID, "sp_dual_step: null problem");
    int64_t m = p->m;
    CHECK_LEN(y, m, "sp_dual_step y");
    CHECK_LEN(ax_bar, m, "sp_dual_step ax_bar");
    CHECK_LEN(y_t, m, "sp_dual_step y_t");
    if (m == 0) return SP_OK;
    k_dual_step<<<grid_for(ctx, m), NT, 0, ctx->stream>>>(y->d, ax_bar->d, p->lc, p->uc, sigma, y_t->d, m);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_halpern_step(sp_ctx *ctx, sp_vec *z, const sp_vec *z_t, const sp_vec *anchor, double w, double rho) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!z) return fail(SP_ERR_INVALID, "sp_halpern_step: null vector");
    CHECK_LEN(z_t, z->n, "sp_halpern_step z_t");
    CHECK_LEN(anchor, z->n, "sp_halpern_step anchor");
    if (z->n == 0) return SP_OK;
    k_halpern<<<grid_for(ctx, z->n), NT, 0, ctx->stream>>>(z->d, z_t->d, anchor->d, w, rho, z->n);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_distance_sq(sp_ctx *ctx, const sp_vec *a, const sp_vec *b, double *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!a || !out) return fail(SP_ERR_INVALID, "sp_distance_sq: null argument");
    CHECK_LEN(b, a->n, "sp_distance_sq b");
    Reduction r(ctx);
    r.add<1>(FDist{a->d, b->d}, a->n);
    return r.finish(out);
}

extern "C" int sp_sub(sp_ctx *ctx, const sp_vec *a, const sp_vec *b, sp_vec *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!a) return fail(SP_ERR_INVALID, "sp_sub: null vector");
    CHECK_LEN(b, a->n, "sp_sub b");
    CHECK_LEN(out, a->n, "sp_sub out");
    if (a->n == 0) return SP_OK;
    k_sub<<<grid_for(ctx, a->n), NT, 0, ctx->stream>>>(a->d, b->d, out->d, a->n);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_norm_sq(sp_ctx *ctx, const sp_vec *v, double *out) { return sp_dot(ctx, v, v, out); }

extern "C" int sp_dot(sp_ctx *ctx, const sp_vec *a, const sp_vec *b, double *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!a || !out) return fail(SP_ERR_INVALID, "sp_dot: null argument");
    CHECK_LEN(b, a->n, "sp_dot b");
    Reduction r(ctx);
    r.add<1>(FDot{a->d, b->d}, a->n);
    return r.finish(out);
}

extern "C" int sp_scale(sp_ctx *ctx, sp_vec *v, double alpha) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!v) return fail(SP_ERR_INVALID, "sp_scale: null vector");
    if (v->n == 0) return SP_OK;
    k_scale<<<grid_for(ctx, v->n), NT, 0, ctx->stream>>>(v->d, alpha, v->n);
    SP_CUDA_TRY(cudaGetLastError());
    return SP_OK;
}

extern "C" int sp_primal_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, const sp_vec *ax,
                               sp_primal_stats_t *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p || !out) return fail(SP_ERR_INVALID, "sp_primal_stats: null argument");
    CHECK_LEN(x, p->n, "sp_primal_stats x");
    CHECK_LEN(ax, p->m, "sp_primal_stats ax");
    Reduction r(ctx);
    r.add<1>(FPrimRes{ax->d, p->lc, p->uc, p->pf}, p->m);
    r.add<1>(FDot{p->c, x->d}, p->n);
    double t[2];
    if ((rc = r.finish(t))) return rc;
    out->residual_sq = t[0];
    out->objective = t[1];
    return SP_OK;
}

extern "C" int sp_dual_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *y, const sp_vec *aty, sp_dual_stats_t *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p || !out) return fail(SP_ERR_INVALID, "sp_dual_stats: null argument");
    CHECK_LEN(y, p->m, "sp_dual_stats y");
    CHECK_LEN(aty, p->n, "sp_dual_stats aty");
    Reduction r(ctx);
    r.add<1>(FDualRows{y->d, p->lc, p->uc}, p->m);
    r.add<2>(FDualCols{p->c, aty->d, p->lv, p->uv, p->df}, p->n);
    double t[3];
    if ((rc = r.finish(t))) return rc;
    out->residual_sq = t[1];
    out->objective = t[0] + t[2];
    return SP_OK;
}

extern "C" int sp_step_dual_residual_sq(sp_ctx *ctx, const sp_problem *p, const sp_vec *x, const sp_vec *x_t,
                                        const sp_vec *aty, const sp_vec *aty_t, double tau, double *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p || !out) return fail(SP_ERR_INVALID, "sp_step_dual_residual_sq: null argument");
    CHECK_LEN(x, p->n, "x");
    CHECK_LEN(x_t, p->n, "x_t");
    CHECK_LEN(aty, p->n, "aty");
    CHECK_LEN(aty_t, p->n, "aty_t");
    Reduction r(ctx);
    r.add<1>(FStepDual{x->d, x_t->d, aty->d, aty_t->d, p->df, 1.0 / tau}, p->n);
    return r.finish(out);
}

extern "C" int sp_primal_ray_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *dx, const sp_vec *adx,
                                   sp_ray_stats_t *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p || !out) return fail(SP_ERR_INVALID, "sp_primal_ray_stats: null argument");
    CHECK_LEN(dx, p->n, "dx");
    CHECK_LEN(adx, p->m, "adx");
    Reduction r(ctx);
    r.add<1>(FPRayRows{adx->d, p->lc, p->uc}, p->m);
    r.add<3>(FPRayCols{dx->d, p->c, p->lv, p->uv}, p->n);
    double t[4];
    if ((rc = r.finish(t))) return rc;
    out->objective = t[3];
    out->violation_sq = t[0] + t[1];
    out->norm_sq = t[2];
    return SP_OK;
}

extern "C" int sp_dual_ray_stats(sp_ctx *ctx, const sp_problem *p, const sp_vec *dy, const sp_vec *atdy,
                                 sp_ray_stats_t *out) {
    int rc = enter(ctx);
    if (rc) return rc;
    if (!p || !out) return fail(SP_ERR_INVALID, "sp_dual_ray_stats: null argument");
    CHECK_LEN(dy, p->m, "dy");
    CHECK_LEN(atdy, p->n, "atdy");
    Reduction r(ctx);
    r.add<3>(FDRayRows{dy->d, p->lc, p->uc}, p->m);
    r.add<2>(FDRayCols{atdy->d, p->lv, p->uv}, p->n);
    double t[5];
    if ((rc = r.finish(t))) return rc;
    out->objective = t[1] + t[4];
    out->violation_sq = t[0] + t[3];
    out->norm_sq = t[2];
    return SP_OK;
}
