// Allocation-free variant of the PDHG stopping-tolerance reduction.
//
// Some callers cannot allocate device memory at the point where they need the
// stopping test: hosts that own the whole device heap themselves (a
// framework's pooled allocator, an inference runtime's plugin enqueue, an
// embedded scanner pipeline that reserves all device memory up front) and
// forbid a library from calling cudaMalloc / cudaFree behind their back.
// tr_tolerance_sums_noalloc serves them: it computes the same FP64 sums as the
// tolerance step inside tr_pdhg_run, but its per-block partial sums live in a
// file-scope __device__ array instead of plan or cudaMalloc memory.
//
// Cost of that choice: every GPU that loads this library holds the array
// (64 KiB) until the process exits; calls share it, so two calls whose
// kernels overlap on the GPU (different streams, no ordering between them)
// race on it and must be serialised by the caller.  Each call writes every
// partial it later reads, so nothing has to be cleared between calls.

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "tr_internal.cuh"

namespace {

constexpr int kNoallocBlocks = 4096;
constexpr int kNoallocThreads = 256;
constexpr int kNoallocItems = 64;   // elements per thread
static_assert((long long)kNoallocBlocks * kNoallocThreads * kNoallocItems == TR_NOALLOC_MAX_ELEMS,
              "header limit and scratch size disagree");

// Per-block (num, den) partial sums: 2 x 4096 doubles = 64 KiB per device.
static __device__ __align__(256) double g_noalloc_partials[2 * kNoallocBlocks];

// Device address of g_noalloc_partials, looked up once per device and
// context: a context that is torn down and re-created (cudaDeviceReset, a host
// that destroys its primary context) reloads the module at a new address, so
// the cached pointer is keyed on the context current at the call.
std::mutex g_mu;
constexpr int kMaxDevices = 64;
double* g_addr[kMaxDevices] = {};
CUcontext g_ctx[kMaxDevices] = {};

// cuCtxGetCurrent from the driver, looked up once (no libcuda link).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(ptr);
    });
    return fn;
}

__global__ void __launch_bounds__(kNoallocThreads) k_tol_partials_noalloc(const float2* __restrict__ cur,
                                                                          const float2* __restrict__ prev,
                                                                          int64_t n, int ref_prev,
                                                                          double* __restrict__ partials) {
    const int64_t base = (int64_t)blockIdx.x * kNoallocThreads * kNoallocItems;
    double num = 0.0, den = 0.0;
#pragma unroll 8
    for (int i = 0; i < kNoallocItems; ++i) {
        const int64_t idx = base + (int64_t)i * kNoallocThreads + threadIdx.x;
        if (idx < n) {
            const float2 c = cur[idx], p = prev[idx];
            const double dx = (double)c.x - (double)p.x, dy = (double)c.y - (double)p.y;
            num += dx * dx + dy * dy;
            const float2 r = ref_prev ? p : c;   // TVMW normalises by the previous iterate
            den += (double)r.x * r.x + (double)r.y * r.y;
        }
    }
    __shared__ double sn[kNoallocThreads / 32], sd[kNoallocThreads / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        num += __shfl_down_sync(0xffffffffu, num, off);
        den += __shfl_down_sync(0xffffffffu, den, off);
    }
    if ((threadIdx.x & 31) == 0) {
        sn[threadIdx.x >> 5] = num;
        sd[threadIdx.x >> 5] = den;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kNoallocThreads / 32; ++w) {
            a += sn[w];
            b += sd[w];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// Fixed-order sum of the partials of this call (blocks [0, nblocks)).
__global__ void k_tol_final_noalloc(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
    __shared__ double sn[256], sd[256];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += partials[2 * i];
        b += partials[2 * i + 1];
    }
    sn[threadIdx.x] = a;
    sd[threadIdx.x] = b;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sn[threadIdx.x] += sn[threadIdx.x + s];
            sd[threadIdx.x] += sd[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sn[0];
        out[1] = sd[0];
    }
}

}  // namespace

extern "C" tr_status tr_tolerance_sums_noalloc(const void* cur, const void* prev, int64_t n, int32_t algorithm,
                                               double* sums_out, void* stream) {
    if (!cur || !prev || !sums_out)
        return tr::fail(TR_ERR_INVALID_ARG, "tr_tolerance_sums_noalloc: null pointer");
    if (algorithm < TR_ALG_TVM || algorithm > TR_ALG_TVMW)
        return tr::fail(TR_ERR_INVALID_ARG, "tr_tolerance_sums_noalloc: unknown algorithm");
    if (n < 0 || n > TR_NOALLOC_MAX_ELEMS)
        return tr::fail(TR_ERR_INVALID_ARG,
                        "tr_tolerance_sums_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                            std::to_string((long long)TR_NOALLOC_MAX_ELEMS) +
                            " complex elements held by its fixed device scratch; use tr_pdhg_run instead");
    int dev = 0;
    TR_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return tr::fail(TR_ERR_UNSUPPORTED, "device ordinal out of range");
    CtxGetCurrentFn get_ctx = ctx_get_current();
    if (!get_ctx) return tr::fail(TR_ERR_CUDA, "tr_tolerance_sums_noalloc: cuCtxGetCurrent unavailable");
    CUcontext ctx = nullptr;   // null until the runtime has made the device's context current
    if (get_ctx(&ctx) != CUDA_SUCCESS) ctx = nullptr;
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!ctx || !g_addr[dev] || g_ctx[dev] != ctx) {
            // set-up, once per device (and again after its context was re-created),
            // with that device current; the lookup also makes the primary context current
            void* ptr = nullptr;
            TR_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_partials));
            if (get_ctx(&ctx) != CUDA_SUCCESS || !ctx)
                return tr::fail(TR_ERR_CUDA, "tr_tolerance_sums_noalloc: no current CUDA context");
            g_addr[dev] = static_cast<double*>(ptr);
            g_ctx[dev] = ctx;
        }
        scratch = g_addr[dev];
    }
    const int64_t per_block = (int64_t)kNoallocThreads * kNoallocItems;
    const int nblocks = (int)std::max<int64_t>(1, (n + per_block - 1) / per_block);
    cudaStream_t st = (cudaStream_t)stream;
    k_tol_partials_noalloc<<<nblocks, kNoallocThreads, 0, st>>>(
        (const float2*)cur, (const float2*)prev, n, algorithm == TR_ALG_TVMW ? 1 : 0, scratch);
    TR_CHECK_LAUNCH();
    k_tol_final_noalloc<<<1, 256, 0, st>>>(scratch, nblocks, sums_out);
    TR_CHECK_LAUNCH();
    return TR_OK;
}
