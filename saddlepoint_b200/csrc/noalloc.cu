// noalloc.cu — sp_dot_noalloc: the dot product aᵀb on caller-owned device memory,
// without allocating anything.
//
// Who needs it: code that cannot call cudaMalloc at the point where it needs a
// reduction — a caller in the middle of CUDA stream capture (allocation is not
// allowed there), a host application whose device memory is all handed out by its
// own pool allocator, or a latency-critical loop that must not hit the implicit
// device synchronisation of cudaMalloc/cudaFree. Such callers hold raw device
// pointers rather than this library's context and vector handles (creating those
// allocates), so the entry point takes plain pointers and a stream.
//
// It is the two-stage reduction of sp_dot: stage one writes one partial sum per
// block, stage two adds the partials in block order into *result. The partials,
// which sp_dot keeps in its context's scratch buffer, live here in a file-scope
// static __device__ array, so every GPU that loads the library holds those 256 KiB
// until the process exits. Stage one uses one block per 2048 elements, so the array
// bounds the length: n may be at most SP_NOALLOC_DOT_MAX_N; longer vectors are
// rejected with SP_ERR_TOO_LARGE before anything is launched.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kPerBlock = 2048;  // elements per stage-one block (8 per thread)
constexpr int kMaxBlocks = 32768;
static_assert((long long)kMaxBlocks * kPerBlock == SP_NOALLOC_DOT_MAX_N, "header and scratch disagree");

// The scratch: one partial sum per stage-one block. Every call overwrites the slots
// it reads before reading them, so nothing has to start at zero.
static __device__ __align__(256) double g_dot_partials[kMaxBlocks];

__global__ void __launch_bounds__(kThreads) k_dot_partials(const double *__restrict__ a, const double *__restrict__ b,
                                                           int64_t n, double *__restrict__ partials) {
    __shared__ double sh[kThreads / 32];
    double s[1] = {0.0};
    const int64_t base = (int64_t)blockIdx.x * kPerBlock;
    for (int i = threadIdx.x; i < kPerBlock; i += kThreads) {
        const int64_t k = base + i;
        if (k < n) s[0] += a[k] * b[k];
    }
    sp::block_sum<1>(s, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kThreads) k_dot_finish(const double *__restrict__ partials, int blocks,
                                                         double *__restrict__ result) {
    __shared__ double sh[kThreads / 32];
    double s[1] = {0.0};
    for (int i = threadIdx.x; i < blocks; i += kThreads) s[0] += partials[i];
    sp::block_sum<1>(s, sh);
    if (threadIdx.x == 0) *result = s[0];
}

// Device address of g_dot_partials, looked up once per device with that device
// current (in host code the symbol's name is only a host-side stand-in).
std::mutex g_mu;
double *g_addr[256] = {};

int scratch_for_current_device(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return SP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_dot_partials) != cudaSuccess || !p) {
            cudaGetLastError();
            return SP_ERR_CUDA;
        }
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return SP_OK;
}

}  // namespace

extern "C" int sp_dot_noalloc(const double *a, const double *b, int64_t n, double *result, void *stream) {
    if (n < 0 || !result || (n > 0 && (!a || !b))) return SP_ERR_INVALID;
    if (n > SP_NOALLOC_DOT_MAX_N) return SP_ERR_TOO_LARGE;
    // an error already pending on this thread belongs to the caller's earlier work:
    // report it without consuming it, and launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) return SP_ERR_CUDA;
    double *partials = nullptr;
    int rc = scratch_for_current_device(&partials);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = n > 0 ? (int)((n + kPerBlock - 1) / kPerBlock) : 1;
    k_dot_partials<<<blocks, kThreads, 0, s>>>(a, b, n, partials);
    if (cudaGetLastError() != cudaSuccess) return SP_ERR_CUDA;
    k_dot_finish<<<1, kThreads, 0, s>>>(partials, blocks, result);
    return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ERR_CUDA;
}
