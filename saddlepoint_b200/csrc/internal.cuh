// internal.cuh — the library's handle types and host helpers shared by the .cu files.
#pragma once

#include <string>

#include "common.cuh"

// Opaque handles of the C ABI.
struct sp_ctx {
    int device = 0;
    int sms = 0;
    int cc_major = 0, cc_minor = 0;
    std::string name;
    std::string last_error;
    cudaStream_t stream = nullptr;
    cudaStream_t aux = nullptr;     // a second stream for set-up work beside `stream`'s
    cudaEvent_t aux_ev = nullptr;   // orders `aux` after work on `stream`
    double *d_partials = nullptr;  // stage-one partials of the trait-method reductions
    double *d_result = nullptr;    // their final values
    double *h_result = nullptr;    // pinned copy read by the host
    int *d_tiles = nullptr;        // work counters of the tile launches on `stream` (tiles.cuh: run_tiles)
};

struct sp_vec {
    sp_ctx *ctx = nullptr;
    double *d = nullptr;
    int64_t n = 0;
};

namespace sp {

// A CSR matrix on the device: int32 indices, FP64 values (+ an FP32 copy for
// the mixed form) and the row-tile plan of tiles.cuh.
struct DevCsr {
    int64_t nrows = 0, ncols = 0, nnz = 0;
    int *rp = nullptr;
    int *ci = nullptr;
    double *v = nullptr;
    float *v32 = nullptr;
    Tile *tiles = nullptr;
    int ntiles = 0;
    uint16_t *sched = nullptr;  // row schedule of every tile (build_schedule)
    int nlong = 0;              // leading tiles that hold one row longer than TILE_NNZ
};

int enter(sp_ctx *ctx);
bool t_ctx_is(const sp_ctx *c);
int upload_csr(sp_ctx *ctx, const sp_csr *h, DevCsr *d, bool want_f32);
void free_csr(DevCsr *d, cudaStream_t st);
// Stream-ordered device memory from the device's pool (see backend.cu): allocated on
// the calling thread's context stream, released on `st`.
int dmalloc(void **p, size_t bytes);
void dfree(void *p, cudaStream_t st);
void keep_pool_memory(int device);
int upload_vec(sp_ctx *ctx, double **d, const double *h, int64_t n);
void launch_spmv(sp_ctx *ctx, const DevCsr &A, const double *x, double *out, cudaStream_t s);

}  // namespace sp

struct sp_problem {
    sp_ctx *ctx = nullptr;
    int64_t m = 0, n = 0;
    sp::DevCsr a, at;
    double *c = nullptr, *lc = nullptr, *uc = nullptr, *lv = nullptr, *uv = nullptr;
    double *pf = nullptr, *df = nullptr;  // primal / dual residual factors
};
