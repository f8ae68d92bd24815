// triplets.cu — CsrMatrix::from_triplets (crates/saddlepoint-core/src/problem.rs:33-77) on
// the GPU, for loading large problems.
//
// This library's rule (and the oracle's): entries grouped by row in input order, each row's
// entries stably sorted by column, runs of one (row, column) summed in input order (the
// first value, then += each next), sums that are exactly zero dropped. The reference sorts
// each row with sort_unstable_by_key (problem.rs:60), which leaves the order of repeated
// (row, column) entries unspecified; the two rules agree bit for bit except where a run of
// three or more repeats of one (row, column) rounds differently in another order. Here: one
// stable radix sort of the key row·ncols + col (a radix sort keeps input order among equal
// keys, so every run comes out in input order), a flag at the head of each run, one thread
// per run summing it in order, a compaction of the non-zero sums, and each row's start found
// by a binary search over the sorted keys. Same entries, same order, same bits as the
// library's host rule.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "internal.cuh"

namespace sp {
namespace {

// Per triplet: its key and its position; *bad set on an index out of range (the reference
// asserts, problem.rs:36).
__global__ void k_trip_keys(const int64_t *__restrict__ rows, const int64_t *__restrict__ cols, int64_t n,
                            int64_t nrows, int64_t ncols, uint64_t *__restrict__ key, int64_t *__restrict__ pos,
                            int *__restrict__ bad) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = rows[t], c = cols[t];
        if (r < 0 || r >= nrows || c < 0 || c >= ncols) {
            *bad = 1;
            key[t] = 0;
        } else {
            key[t] = (uint64_t)r * (uint64_t)ncols + (uint64_t)c;
        }
        pos[t] = t;
    }
}

// 1 at the first entry of each run of equal keys.
__global__ void k_trip_heads(const uint64_t *__restrict__ skey, int64_t n, int *__restrict__ head) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        head[t] = (t == 0 || skey[t] != skey[t - 1]) ? 1 : 0;
}

// One thread per run: its sum in input order, its key, and whether the sum is kept.
__global__ void k_trip_sums(const uint64_t *__restrict__ skey, const int64_t *__restrict__ spos,
                            const double *__restrict__ vals, const int64_t *__restrict__ start, const int *nrun,
                            int64_t n, uint64_t *__restrict__ rkey, double *__restrict__ rval, int *__restrict__ keep) {
    const int64_t runs = *nrun;
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < runs; s += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = start[s], b = s + 1 < runs ? start[s + 1] : n;
        double sum = vals[spos[a]];
        for (int64_t k = a + 1; k < b; ++k) sum += vals[spos[k]];
        rkey[s] = skey[a];
        rval[s] = sum;
        keep[s] = sum != 0.0;
    }
}

// Each row's first entry among the kept, sorted keys; and the column of every entry.
__global__ void k_trip_csr(const uint64_t *__restrict__ fkey, int64_t nnz, int64_t nrows, int64_t ncols,
                           int64_t *__restrict__ rp, int32_t *__restrict__ ci) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nrows; i += stride) {
        const uint64_t first = (uint64_t)i * (uint64_t)ncols;
        int64_t lo = 0, hi = nnz;
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (fkey[mid] < first) lo = mid + 1;
            else hi = mid;
        }
        rp[i] = i == nrows ? nnz : lo;
    }
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += stride)
        ci[k] = (int32_t)(fkey[k] % (uint64_t)ncols);
}

struct OwnedCsr {
    std::vector<int64_t> rp;
    std::vector<int32_t> ci;
    std::vector<double> v;
};
std::map<const void *, OwnedCsr *> g_csr;
std::mutex g_csr_mu;

}  // namespace
}  // namespace sp

extern "C" int sp_csr_from_triplets(sp_ctx *ctx, int64_t nrows, int64_t ncols, int64_t ntrip, const int64_t *rows,
                                    const int64_t *cols, const double *vals, sp_csr *out) {
    using namespace sp;
    int rc = enter(ctx);
    if (rc) return rc;
    if (!out || nrows < 0 || ncols < 0 || ntrip < 0 || (ntrip > 0 && (!rows || !cols || !vals)))
        return fail(SP_ERR_INVALID, "sp_csr_from_triplets: bad argument");
    if (nrows > INT32_MAX - 1 || ncols > INT32_MAX - 1 || ntrip > INT32_MAX - 1)
        return fail(SP_ERR_TOO_LARGE, "sp_csr_from_triplets: problem too large for 32-bit sparse indices");
    memset(out, 0, sizeof *out);
    auto *o = new OwnedCsr();
    o->rp.assign(nrows + 1, 0);
    cudaStream_t st = ctx->stream;
    std::vector<void *> bufs;
    auto release = [&] {
        for (void *p : bufs) dfree(p, st);
        cudaStreamSynchronize(st);
    };
    auto alloc = [&](void **p, size_t bytes) {
        const int r = dmalloc(p, std::max<size_t>(bytes, 16));
        if (!r) bufs.push_back(*p);
        return r;
    };
    int64_t nnz = 0;
    if (ntrip > 0) {
        int64_t *d_rows, *d_cols, *pos, *spos, *start;
        double *d_vals, *rval, *fval;
        uint64_t *key, *skey, *rkey, *fkey;
        int *bad, *head, *nrun, *keep, *nkeep;
        const size_t n = (size_t)ntrip;
        if ((rc = alloc((void **)&d_rows, 8 * n)) || (rc = alloc((void **)&d_cols, 8 * n)) ||
            (rc = alloc((void **)&d_vals, 8 * n)) || (rc = alloc((void **)&key, 8 * n)) ||
            (rc = alloc((void **)&skey, 8 * n)) || (rc = alloc((void **)&pos, 8 * n)) ||
            (rc = alloc((void **)&spos, 8 * n)) || (rc = alloc((void **)&head, 4 * n)) ||
            (rc = alloc((void **)&start, 8 * n)) || (rc = alloc((void **)&rkey, 8 * n)) ||
            (rc = alloc((void **)&rval, 8 * n)) || (rc = alloc((void **)&keep, 4 * n)) ||
            (rc = alloc((void **)&fkey, 8 * n)) || (rc = alloc((void **)&fval, 8 * n)) ||
            (rc = alloc((void **)&bad, 4)) || (rc = alloc((void **)&nrun, 4)) || (rc = alloc((void **)&nkeep, 4))) {
            release();
            delete o;
            return rc;
        }
        auto cuda_fail = [&](cudaError_t e) {
            release();
            delete o;
            return fail(SP_ERR_CUDA, std::string("sp_csr_from_triplets: ") + cudaGetErrorString(e));
        };
        cudaError_t e;
        if ((e = cudaMemcpyAsync(d_rows, rows, 8 * n, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(d_cols, cols, 8 * n, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(d_vals, vals, 8 * n, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemsetAsync(bad, 0, 4, st)))
            return cuda_fail(e);
        const int g = std::max(1, std::min<int>((int)((ntrip + NT - 1) / NT), ctx->sms * 16));
        k_trip_keys<<<g, NT, 0, st>>>(d_rows, d_cols, ntrip, nrows, ncols, key, pos, bad);
        int end_bit = 1;
        const uint64_t maxkey = (uint64_t)std::max<int64_t>(nrows, 1) * (uint64_t)std::max<int64_t>(ncols, 1);
        while (end_bit < 64 && (maxkey >> end_bit)) ++end_bit;
        thrust::counting_iterator<int64_t> idx(0);
        size_t b0 = 0, b1 = 0, b2 = 0;
        if ((e = cub::DeviceRadixSort::SortPairs(nullptr, b0, key, skey, pos, spos, ntrip, 0, end_bit, st)) ||
            (e = cub::DeviceSelect::Flagged(nullptr, b1, idx, head, start, nrun, ntrip, st)) ||
            (e = cub::DeviceSelect::Flagged(nullptr, b2, rkey, keep, fkey, nkeep, ntrip, st)))
            return cuda_fail(e);
        void *tmp;
        if ((rc = alloc(&tmp, std::max({b0, b1, b2})))) {
            release();
            delete o;
            return rc;
        }
        if ((e = cub::DeviceRadixSort::SortPairs(tmp, b0, key, skey, pos, spos, ntrip, 0, end_bit, st))) return cuda_fail(e);
        k_trip_heads<<<g, NT, 0, st>>>(skey, ntrip, head);
        if ((e = cub::DeviceSelect::Flagged(tmp, b1, idx, head, start, nrun, ntrip, st))) return cuda_fail(e);
        // flags past the last run stay 0: the selections below run over all ntrip slots
        if ((e = cudaMemsetAsync(keep, 0, 4 * n, st))) return cuda_fail(e);
        k_trip_sums<<<g, NT, 0, st>>>(skey, spos, d_vals, start, nrun, ntrip, rkey, rval, keep);
        // the kept runs' keys and values, in order
        if ((e = cub::DeviceSelect::Flagged(tmp, b2, rkey, keep, fkey, nkeep, ntrip, st)) ||
            (e = cub::DeviceSelect::Flagged(tmp, b2, rval, keep, fval, nkeep, ntrip, st)))
            return cuda_fail(e);
        int hbad = 0, hkeep = 0;
        if ((e = cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st)) ||
            (e = cudaMemcpyAsync(&hkeep, nkeep, 4, cudaMemcpyDeviceToHost, st)) || (e = cudaStreamSynchronize(st)))
            return cuda_fail(e);
        if (hbad) {
            release();
            delete o;
            return fail(SP_ERR_INVALID, "sp_csr_from_triplets: a row or column index is out of range");
        }
        nnz = hkeep;
        int64_t *rp;
        int32_t *ci;
        if ((rc = alloc((void **)&rp, 8 * (size_t)(nrows + 1))) || (rc = alloc((void **)&ci, 4 * (size_t)nnz))) {
            release();
            delete o;
            return rc;
        }
        const int gr = std::max(1, std::min<int>((int)((std::max<int64_t>(nrows + 1, nnz) + NT - 1) / NT), ctx->sms * 16));
        k_trip_csr<<<gr, NT, 0, st>>>(fkey, nnz, nrows, ncols, rp, ci);
        o->ci.resize(nnz);
        o->v.resize(nnz);
        if ((e = cudaMemcpyAsync(o->rp.data(), rp, 8 * (size_t)(nrows + 1), cudaMemcpyDeviceToHost, st)) ||
            (nnz && (e = cudaMemcpyAsync(o->ci.data(), ci, 4 * (size_t)nnz, cudaMemcpyDeviceToHost, st))) ||
            (nnz && (e = cudaMemcpyAsync(o->v.data(), fval, 8 * (size_t)nnz, cudaMemcpyDeviceToHost, st))) ||
            (e = cudaStreamSynchronize(st)))
            return cuda_fail(e);
        release();
    }
    o->ci.reserve(1);  // every pointer valid for an empty matrix
    o->v.reserve(1);
    out->nrows = nrows;
    out->ncols = ncols;
    out->nnz = nnz;
    out->row_ptr = o->rp.data();
    out->col_idx = o->ci.data();
    out->values = o->v.data();
    std::lock_guard<std::mutex> lock(g_csr_mu);
    g_csr[out->row_ptr] = o;
    return SP_OK;
}

extern "C" void sp_csr_release(sp_csr *m) {
    using namespace sp;
    if (!m || !m->row_ptr) return;
    OwnedCsr *o = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_csr_mu);
        auto it = g_csr.find(m->row_ptr);
        if (it == g_csr.end()) return;  // not one of this library's
        o = it->second;
        g_csr.erase(it);
    }
    delete o;
    memset(m, 0, sizeof *m);
}
