// Internal definitions shared by the toporecon_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "toporecon_b200.h"

namespace tr {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
tr_status fail(tr_status code, const std::string& msg);
tr_status cuda_fail(cudaError_t err, const char* what, const char* file, int line);

#define TR_CUDA(expr)                                                   \
    do {                                                                \
        cudaError_t _e = (expr);                                        \
        if (_e != cudaSuccess) return ::tr::cuda_fail(_e, #expr, __FILE__, __LINE__); \
    } while (0)

#define TR_CHECK_LAUNCH() TR_CUDA(cudaGetLastError())

#define TR_TRY(expr)                                                    \
    do {                                                                \
        tr_status _s = (expr);                                          \
        if (_s != TR_OK) return _s;                                     \
    } while (0)

// Makes a plan's device current for the lifetime of the guard and restores the
// caller's device afterwards.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// ------------------------------------------------------------------ device error word
// Kernels that wait on hardware (mbarrier polls) give up after the plan's poll
// limit (kMbarPollLimit unless tr_plan_set_wait_limit changed it), wait at most
// kMbarDrainLimit more polls for their own copies in flight, set a bit here and
// leave; the host reads the word with the tolerance scalars.
constexpr int kMbarPollLimit = 1 << 20;
constexpr int kMbarDrainLimit = 1 << 20;
constexpr int kDevErrTmaWait = 1;
constexpr int kDevErrCluster = 2;   // a cluster kernel ran without the cluster shape it needs (no work done)

// ------------------------------------------------------------------ complex helpers
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// Packed f32x2 complex arithmetic (sm_100 add/sub/mul/fma.rn.f32x2): each
// instruction rounds both components exactly like the scalar operation, so
// results match scalar IEEE code op for op; host builds use the scalar forms.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
__device__ __forceinline__ unsigned long long f2_pack(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long r) {
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(r));
    return d;
}
#endif
// a + b
__host__ __device__ __forceinline__ float2 cadd_p(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(b)));
    return f2_unpack(r);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}
// a - b
__host__ __device__ __forceinline__ float2 csub_p(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_pack(a)), "l"(f2_pack(b)));
    return f2_unpack(r);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// c + w * v (real w on both components)
__host__ __device__ __forceinline__ float2 cfma_real(float w, float2 v, float2 c) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2_pack(make_float2(w, w))), "l"(f2_pack(v)), "l"(f2_pack(c)));
    return f2_unpack(r);
#else
    return make_float2(fmaf(w, v.x, c.x), fmaf(w, v.y, c.y));
#endif
}
// a * b as a.x * (b.x, b.y) + a.y * (-b.y, b.x): one packed multiply, one packed FMA
__host__ __device__ __forceinline__ float2 cmul_p(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
    unsigned long long t, r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(f2_pack(make_float2(a.y, a.y))), "l"(f2_pack(make_float2(-b.y, b.x))));
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(f2_pack(make_float2(a.x, a.x))), "l"(f2_pack(b)), "l"(t));
    return f2_unpack(r);
#else
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
#endif
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }

// ------------------------------------------------------------------ FFT plan
constexpr int kMaxStages = 12;
constexpr int kMaxFftLen = 1024;

struct FftAxis {
    int n = 0;        // image length along the axis
    int L = 0;        // oversampled (transform) length
    int h = 0;        // centre shift L/2
    int pad = 0;      // centred zero-pad offset L/2 - n/2
    int nstages = 0;
    int radix[kMaxStages] = {0};
    float2* twiddle = nullptr;   // device [L]: exp(-2 pi i k / L)
    float* apod = nullptr;       // device [n]: per-axis de-apodisation
};

// Per-launch description of the stage sequence, passed by value.
struct FftStages {
    int L;
    int nstages;
    int radix[kMaxStages];
};

inline FftStages stages_of(const FftAxis& a) {
    FftStages s;
    s.L = a.L;
    s.nstages = a.nstages;
    for (int i = 0; i < kMaxStages; ++i) s.radix[i] = a.radix[i];
    return s;
}

// ------------------------------------------------------------------ plan
struct Bin {
    int64_t offset = 0;   // first sample of the bin in the concatenated arrays
    int64_t count = 0;
    int64_t list_offset = 0;   // first gather-list entry of the bin
    int64_t list_count = 0;
    int64_t n_busy = 0;        // grid tiles with at least one gather-list entry
    int64_t n_zero = 0;        // empty tiles in occupied (y, x) tile columns (zero-filled by gridding)
    int64_t n_occ_cols = 0;    // occupied (y, x) tile columns
    int64_t work_offset = 0;   // first gridding work item of the bin
    int64_t n_work = 0;        // work items: busy tiles, the heaviest split into list ranges
    int64_t split_offset = 0;  // first split-tile record of the bin
    int64_t n_split = 0;       // tiles whose list is split over several work items
};

struct PdhgGraph;        // defined in tr_pdhg.cu
struct WaveletPlan;      // defined in tr_wavelet.cu

}  // namespace tr

struct tr_plan {
    int device = 0;
    int n[3] = {0, 0, 0};     // Z, Y, X
    int os[3] = {0, 0, 0};
    int C = 1, E = 1, B = 1;
    float beta = 0.f;
    int width = 4;
    float fwd_scale = 1.f;    // 1 / (sqrt(N) * w^3)
    float adj_scale = 1.f;    // 1 / (sqrt(N) * w^3)
    tr::FftAxis ax[3];
    std::vector<tr::Bin> bins;
    int64_t total = 0;
    // device-resident trajectory (tile-sorted per bin)
    float4* ks = nullptr;        // (kz, ky, kx, dcf) in oversampled-grid units, sorted
    void* taps = nullptr;        // per-sample first taps and KB weights (TapRec), sorted
    int32_t* perm = nullptr;     // sorted position -> acquisition index within the bin
    int2* glist = nullptr;          // gridding gather lists: (sample in bin, packed tap offsets), all bins
    int32_t* list_start = nullptr;  // per bin [ntiles + 1] (relative to the bin's first entry)
    int32_t* tile_order = nullptr;  // per bin [ntiles]: busy tiles heaviest first, then the empty tiles of
                                    // occupied columns, then those of unoccupied columns
    uint8_t* colmask = nullptr;     // per bin [ntile[1] * ntile[2]]: 1 where some tile of the (y, x) column is busy
    bool skip_empty_cols = true;    // z passes skip unoccupied columns (not TR_PLAN_NO_COLUMN_SKIP, not fused y + z)
    int4* work = nullptr;           // gridding work items (tile, first entry, end entry, partial slot or -1)
    int4* splits = nullptr;         // split tiles (tile, first partial slot, partial count, 0)
    int ntile[3] = {0, 0, 0};
    int64_t ntiles = 0;
    bool has_dcf = false;
    // coil maps (Z, Y, X, C) interleaved
    float2* maps = nullptr;
    // NUFFT workspace
    float2* bufA = nullptr;      // >= OSZ*OSY*OSX*ncol (grid / x-pass output)
    float2* bufB = nullptr;      // >= Z*OSY*OSX*ncol  (y-pass output / z-pass adjoint output)
    size_t buf_cols = 0;         // ncol the buffers are sized for
    // single-image drop-in scratch
    float2* one_in = nullptr;
    float2* one_out = nullptr;
    size_t one_elems = 0;
    // reductions
    double* partials = nullptr;
    int npartials = 0;
    double* tol_dev = nullptr;   // [4]
    double* tol_host = nullptr;  // pinned [4]
    int* dev_err = nullptr;      // device error word (kDevErr* bits)
    int poll_limit = tr::kMbarPollLimit;   // polls before a bounded mbarrier wait gives up
    int* err_host = nullptr;     // pinned copy, refreshed with the tolerance scalars
    // launch shapes
    int line_width = 16;
    int spread_cols = 128;       // most k-space columns per gridding CTA
    bool use_tma = true;
    bool fuse_yz = false;        // TR_PLAN_YZ_FUSION: fused y + z passes where the geometry allows
    bool two_pass_320 = true;    // 320-point TMA FFT passes in two shared-memory passes (not TR_PLAN_THREE_PASS_320)
    bool autotune = false;       // TR_PLAN_AUTOTUNE: time launch-shape candidates on first use
    std::map<int, int> spread_cols_tuned;   // column count -> chosen spread_cols         // TMA-tiled FFT passes where the geometry allows
    // TVMW
    tr::WaveletPlan* wav = nullptr;
    // CUDA graph of one PDHG iteration
    tr::PdhgGraph* graph = nullptr;
    int64_t workspace_bytes = 0;
};

namespace tr {

tr_status ensure_nufft_buffers(tr_plan* p, size_t ncol);
tr_status nufft_forward_cols(tr_plan* p, int bin, const float2* images, int64_t img_stride, int n_img,
                             const float2* maps, int C, int mode, float sigma, const float2* y,
                             float2* out, cudaStream_t st);
tr_status nufft_adjoint_cols(tr_plan* p, int bin, const float2* ksp, int n_img, const float2* maps, int C,
                             bool use_dcf, float2* images, int64_t img_stride, cudaStream_t st);
tr_status wavelet_prepare(tr_plan* p);
tr_status wavelet_dual(tr_plan* p, const float2* u_bar, float2* p_w2, float sigma, float lam, cudaStream_t st);
tr_status wavelet_adjoint(tr_plan* p, const float2* p_w2, float2* out, cudaStream_t st);
void wavelet_destroy(tr_plan* p);
void wavelet_info(const tr_plan* p, int32_t* levels, int64_t* coeffs);
void pdhg_destroy(tr_plan* p);

// forward interpolation output modes
constexpr int kInterpStore = 0;     // out = A x
constexpr int kInterpDualProx = 1;  // out = (out + sigma (A x - y)) / (1 + sigma)

}  // namespace tr
