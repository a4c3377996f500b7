// pcf_noalloc.cu -- an allocation-free variant of the deterministic global
// dot product (pcf_global_dot).
//
// pcf_global_dot keeps its per-block partial sums in device memory that the
// handle allocates.  Some callers cannot let a library allocate device memory:
// a host model whose GPU memory is owned by its own pool allocator (Julia's
// CUDA.jl pool, for example, which may hold nearly all of the device), or a
// time step that is being recorded into a CUDA graph, where cudaMalloc and
// cudaFree are not permitted and would also synchronise the device.  This
// entry point takes only the caller's device buffers and keeps its scratch
// (the partial sums and the last-block ticket) in a file-scope __device__
// array of fixed size, which every GPU that loads the library holds until
// the process exits.
#include <cuda.h>

#include <mutex>

#include "pcf_internal.cuh"

namespace {

// Sum over a block of 256 threads (result in thread 0), fixed order.
__device__ __forceinline__ double block_sum256(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    v = 0.0;
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

constexpr int kNoallocBlocks = 8192;        // partial sums held in the scratch array (64 KB)
constexpr long long kNoallocChunk = 32768;  // elements summed by one block
constexpr long long kNoallocMaxN = (long long)kNoallocBlocks * kNoallocChunk;  // 268,435,456 elements

struct NoallocScratch {
    double partials[kNoallocBlocks];
    unsigned int ticket;
};

// The scratch: one instance per device, shared by every call.
__device__ __align__(256) NoallocScratch g_noalloc_scratch;

// One block per chunk of kNoallocChunk elements; each block writes its partial
// sum, and the last block to finish adds the partials in block order, so the
// result does not depend on scheduling.
__global__ void __launch_bounds__(256) k_dot_noalloc(const double *__restrict__ a, const double *__restrict__ b,
                                                    long long n, NoallocScratch *s, double *out) {
    __shared__ double sh[32];
    __shared__ int is_last;
    const long long lo = (long long)blockIdx.x * kNoallocChunk;
    const long long hi = lo + kNoallocChunk < n ? lo + kNoallocChunk : n;
    double v = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) v += a[i] * b[i];
    v = block_sum256(v, sh);
    if (threadIdx.x == 0) {
        s->partials[blockIdx.x] = v;
        __threadfence();
        const unsigned t = atomicAdd(&s->ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double acc = 0.0;
    for (unsigned q = threadIdx.x; q < gridDim.x; q += blockDim.x) acc += __ldcg(s->partials + q);
    acc = block_sum256(acc, sh);
    if (threadIdx.x == 0) {
        *out = acc;
        s->ticket = 0u;
    }
}

std::mutex g_noalloc_mutex;
NoallocScratch *g_noalloc_ptr[64] = {};
CUcontext g_noalloc_ctx[64] = {};

// The driver's cuCtxGetCurrent, resolved once through the runtime (the
// library does not link libcuda), or null if it cannot be resolved.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<CtxGetCurrentFn>(nullptr);
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    return fn;
}

// Device address of the scratch array for the current device.  In host code
// the symbol g_noalloc_scratch is only a host-side stand-in, so the address is
// looked up with cudaGetSymbolAddress on the first call on a device, and again
// whenever the device's current context has changed (after a
// cudaDeviceReset the module is loaded anew and the old address is stale).
int noalloc_scratch(NoallocScratch **p) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return PCF_ENODEVICE;
    CUcontext ctx = nullptr;
    if (CtxGetCurrentFn f = ctx_get_current()) f(&ctx);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev] || g_noalloc_ctx[dev] != ctx) {
        void *q = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&q, g_noalloc_scratch);
        if (e != cudaSuccess) return pcf_set_cuda_error(e);
        g_noalloc_ptr[dev] = static_cast<NoallocScratch *>(q);
        // the context is current only once the runtime has set it up
        if (CtxGetCurrentFn f = ctx_get_current()) f(&ctx);
        g_noalloc_ctx[dev] = ctx;
    }
    *p = g_noalloc_ptr[dev];
    return PCF_OK;
}

}  // namespace

extern "C" int pcf_global_dot_noalloc(const double *a, const double *b, long long n, double *result,
                                      void *stream) {
    if (!result || n < 0 || (n > 0 && (!a || !b))) return PCF_EINVAL;
    if (n > kNoallocMaxN) return PCF_ERANGE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NoallocScratch *s = nullptr;
    int rc = noalloc_scratch(&s);
    if (rc) return rc;
    if (n == 0) {
        PCF_CUDA_TRY(cudaMemsetAsync(result, 0, sizeof(double), st));
        return PCF_OK;
    }
    // the ticket must start at zero; a previous call leaves it at zero, but a
    // call that never finished (an aborted context) would not
    PCF_CUDA_TRY(cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned int), st));
    const unsigned blocks = (unsigned)((n + kNoallocChunk - 1) / kNoallocChunk);
    k_dot_noalloc<<<blocks, 256, 0, st>>>(a, b, n, s, result);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}
