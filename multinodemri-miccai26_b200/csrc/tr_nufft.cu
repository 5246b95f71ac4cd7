// Kaiser-Bessel NUFFT for sm_100a: plan (tile sort), fused FFT passes,
// interpolation and deterministic tile-gather gridding, and their C ABI.
//
// Numerical definition (the reference's SigPy 0.1.27 defaults, called at
// src/toporecon/nufft_backend.py:104-107 and :112-116):
//   forward  y = I_KB( FFTc( pad( apod . x ) ) ) / (sqrt(N) w^3)
//   adjoint  x = apod . crop( IFFTc( G_KB(y) ) ) / (sqrt(N) w^3)
// with oversampling 1.25, width w = 4, beta = pi sqrt((w/os (os - 0.5))^2 - 0.8),
// taps ceil(k - 2) .. floor(k + 2) per axis and periodic wrap.
//
// Data layout (device):
//   images           (n_img, Z, Y, X)                  complex64
//   coil maps        (Z, Y, X, C)                      complex64, plan-owned copy
//   x-pass buffer    (Z, Y, OSX, ncol)                 ncol = n_img * C columns
//   y-pass buffer    (Z, OSY, OSX, ncol)
//   grid             (OSZ, OSY, OSX, ncol)
//   k-space          (M_b, ncol) per bin, tile-sorted samples
// The trajectory of each bin is sorted by 4x4x4 grid tile (stable counting
// sort on the host, so the gather order and hence every sum is deterministic).

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "tr_fft.cuh"
#include "tr_internal.cuh"

namespace tr {

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

tr_status fail(tr_status code, const std::string& msg) {
    set_error(msg);
    return code;
}

tr_status cuda_fail(cudaError_t err, const char* what, const char* file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)err, cudaGetErrorString(err), what,
             file, line);
    set_error(buf);
    return err == cudaErrorMemoryAllocation ? TR_ERR_OOM : TR_ERR_CUDA;
}

// ------------------------------------------------------------------ KB window
// Modified Bessel I0 by the Abramowitz & Stegun 9.8.1 / 9.8.2 approximations
// (the same published formulas SigPy evaluates), then the unnormalised window.
__host__ __device__ __forceinline__ float bessel_i0_as(float x) {
    if (x < 3.75f) {
        float t = x * (1.0f / 3.75f);
        float t2 = t * t;
        return 1.0f + t2 * (3.5156229f + t2 * (3.0899424f + t2 * (1.2067492f +
               t2 * (0.2659732f + t2 * (0.0360768f + t2 * 0.0045813f)))));
    }
    float u = 3.75f / x;
    float poly = 0.39894228f + u * (0.01328592f + u * (0.00225319f + u * (-0.00157565f + u * (0.00916281f +
                 u * (-0.02057706f + u * (0.02635537f + u * (-0.01647633f + u * 0.00392377f)))))));
    return expf(x) * rsqrtf(x) * poly;
}

__device__ __forceinline__ float kb_weight(float d, float beta) {
    // d = (tap - k) / (w / 2); zero outside |d| <= 1
    if (fabsf(d) > 1.0f) return 0.0f;
    return bessel_i0_as(beta * sqrtf(fmaxf(1.0f - d * d, 0.0f)));
}

__device__ __forceinline__ int pmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// First tap and the five candidate weights of one axis (w = 4).
__device__ __forceinline__ int axis_taps(float k, float beta, float (&w)[5]) {
    // ceil(k - w/2) evaluated in double like the reference's tap bounds
    const int b0 = (int)ceil((double)k - 2.0);
#pragma unroll
    for (int t = 0; t < 5; ++t) w[t] = kb_weight(((float)(b0 + t) - k) * 0.5f, beta);
    return b0;
}

// ------------------------------------------------------------------ forward x pass
// One CTA: `rows` consecutive (z, y) image rows x `cc` coils of one image.
// Fuses: image * coil map * separable apodisation * scale, centred zero-pad,
// x FFT, centred shift; output into the (Z, Y, OSX, ncol) buffer.
struct FwdXArgs {
    const float2* img;      // (n_img, Z, Y, X)
    int64_t img_stride;
    const float2* maps;     // (Z, Y, X, C) or null
    int C;                  // coils per image (1 when maps == null)
    int n_img;
    int Z, Y, X, OSX, h, pad;
    int rows, cc;           // rows per CTA, coils per CTA
    const float* apz;
    const float* apy;
    const float* apx;
    float scale;
    const float2* tw;
    FftStages S;
    float2* out;            // (Z, Y, OSX, ncol)
    int ncol;
    int* err;               // device error word (kDevErr* bits)
    int poll;               // polls before a bounded mbarrier wait gives up
};

__global__ void __launch_bounds__(256) k_fwd_x(FwdXArgs a) {
    extern __shared__ float2 sm[];
    const int W = a.rows * a.cc;
    const int L = a.S.L;
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);      // images of one row block run side by side
    const int row0 = (int)(blockIdx.x / (unsigned)a.n_img) * a.rows;
    const int c0 = blockIdx.z * a.cc;
    const int nrows = a.Z * a.Y;
    const float2* __restrict__ src = a.img + (int64_t)img * a.img_stride;
    for (int i = threadIdx.x; i < L; i += blockDim.x) tws[i] = a.tw[i];
    // fill: smA[m][w] = image * map * apodisation * scale at padded, shifted position m
    const int total = L * W;
#pragma unroll 4
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int m = idx / W, w = idx - m * W;
        const int rl = w / a.cc, cl = w - rl * a.cc;
        const int row = row0 + rl, c = c0 + cl;
        int j = m + a.h;
        if (j >= L) j -= L;
        const int x = j - a.pad;
        float2 v = make_float2(0.f, 0.f);
        if (x >= 0 && x < a.X && row < nrows && c < a.C) {
            const int z = row / a.Y, y = row - z * a.Y;
            v = src[(int64_t)row * a.X + x];
            if (a.maps) v = cmul(v, a.maps[((int64_t)row * a.X + x) * a.C + c]);
            v = cscale(v, a.apz[z] * a.apy[y] * a.apx[x] * a.scale);
        }
        smA[idx] = v;
    }
    __syncthreads();
    auto load = [smA, W](int m, int w) -> float2 { return smA[m * W + w]; };
    auto store = [&](int k, int w, float2 v) {
        const int rl = w / a.cc, cl = w - rl * a.cc;
        const int row = row0 + rl;
        const int c = c0 + cl;
        if (row >= nrows || c >= a.C) return;
        int g = k + a.h;
        if (g >= L) g -= L;
        a.out[((int64_t)row * a.OSX + g) * a.ncol + (int64_t)img * a.C + c] = v;
    };
    fft_run(smA, smB, tws, a.S, W, false, load, store);
}

// ------------------------------------------------------------------ generic line pass
// Data viewed as [outer][rows][inner]; transforms along rows for W consecutive
// inner elements per CTA.  Input rows present: Lin (pad offset p_in inside the
// length-L line); output rows kept: Lout (crop offset p_out).
struct LineArgs {
    const float2* in;
    float2* out;
    int64_t inner;
    int Lin, Lout, p_in, p_out, h;
    int W;
    int vec16;              // rows are 16-byte aligned: copy two elements per cp.async
    bool inv;
    const float2* tw;
    FftStages S;
    int* err;               // device error word (kDevErr* bits)
    int poll;               // polls before a bounded mbarrier wait gives up
    int kA, kB;             // TMA variant: first transform row of each output box
    // z passes: (y, x) tile columns that no sample's kernel reaches; null: none skipped
    const uint8_t* colmask; // [nt1 * nt2] 1: occupied
    int skip_zero;          // 0: a CTA whose lines are all unoccupied returns (forward: the output is never
                            // read); 1: it writes zeros to its output rows (adjoint: the lines are zero)
    int mcol, mosx, mnt2;   // k-space columns, OSX and tile columns along x of the mask
};

// Empty-column skip of the z passes.  Inner index q of a z pass is
// ((y OSX + x) ncol + column); a line is unoccupied when the tile column
// (y / 4, x / 4) holds no busy tile: gridding wrote no tile there (the line is
// all zeros) and interpolation reads no tap there.  True when every line
// q0 .. q0 + W - 1 (< inner) of the CTA is unoccupied (the same for all threads).
// The host passes a mask only when W divides ncol, so a CTA never mixes lines
// of occupied and unoccupied columns (it would read unwritten tiles).
__device__ __forceinline__ bool lines_unoccupied(const LineArgs& a, int64_t q0, int W) {
    if (!a.colmask) return false;
    const int64_t q1 = min(q0 + W, a.inner) - 1;
    for (int64_t yx = q0 / a.mcol; yx <= q1 / a.mcol; ++yx) {
        const int y = (int)(yx / a.mosx), x = (int)(yx - (int64_t)y * a.mosx);
        if (a.colmask[(y >> 2) * a.mnt2 + (x >> 2)]) return false;
    }
    return true;
}
// The zeros of an unoccupied CTA's output rows (adjoint z pass): [Lout][W] at q0.
__device__ __forceinline__ void lines_write_zeros(const LineArgs& a, int64_t q0, int W, int64_t outer) {
    float2* out = a.out + outer * a.Lout * a.inner;
    for (int i = threadIdx.x; i < a.Lout * W; i += blockDim.x) {
        const int o = i / W, w = i - o * W;
        if (q0 + w < a.inner) out[(int64_t)o * a.inner + q0 + w] = make_float2(0.f, 0.f);
    }
}

// The CTA's [L][W] tile is staged with cp.async (every load in flight at
// once, zero-filled pad rows and tail columns), then all stages run from
// shared memory and the last stage stores straight to global memory.
__global__ void __launch_bounds__(256) k_line(LineArgs a) {
    extern __shared__ float2 sm[];
    const int W = a.W;
    const int L = a.S.L;
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int64_t q0 = (int64_t)blockIdx.x * W;
    if (lines_unoccupied(a, q0, W)) {
        if (a.skip_zero) lines_write_zeros(a, q0, W, blockIdx.y);
        return;
    }
    const int64_t outer = blockIdx.y;
    const float2* __restrict__ in = a.in + outer * a.Lin * a.inner;
    float2* __restrict__ out = a.out + outer * a.Lout * a.inner;
    for (int i = threadIdx.x; i < L; i += blockDim.x) tws[i] = a.tw[i];
    if (a.vec16) {
        const int nch = W >> 1;
        for (int idx = threadIdx.x; idx < L * nch; idx += blockDim.x) {
            const int m = idx / nch, ch = idx - m * nch;
            int j = m + a.h;
            if (j >= L) j -= L;
            const int i = j - a.p_in;
            const int64_t q = q0 + 2 * ch;
            int bytes = 0;
            const float2* g = a.in;
            if (i >= 0 && i < a.Lin && q < a.inner) {
                bytes = (q + 1 < a.inner) ? 16 : 8;
                g = in + (int64_t)i * a.inner + q;
            }
            cp_async16(smA + m * W + 2 * ch, g, bytes);
        }
    } else {
        for (int idx = threadIdx.x; idx < L * W; idx += blockDim.x) {
            const int m = idx / W, w = idx - m * W;
            int j = m + a.h;
            if (j >= L) j -= L;
            const int i = j - a.p_in;
            const int64_t q = q0 + w;
            int bytes = 0;
            const float2* g = a.in;
            if (i >= 0 && i < a.Lin && q < a.inner) {
                bytes = 8;
                g = in + (int64_t)i * a.inner + q;
            }
            cp_async8(smA + idx, g, bytes);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    auto load = [smA, W](int m, int w) -> float2 { return smA[m * W + w]; };
    auto store = [&](int k, int w, float2 v) {
        const int64_t q = q0 + w;
        int o = k + a.h - a.p_out;
        o %= L;
        if (o < 0) o += L;
        if (q >= a.inner || o >= a.Lout) return;
        out[(int64_t)o * a.inner + q] = v;
    };
    fft_run(smA, smB, tws, a.S, W, a.inv, load, store);
}

// ------------------------------------------------------------------ adjoint x pass
// One CTA: `rows` rows x all C coils of one image (coils processed in chunks
// of `cc`).  Fuses: x IFFT, centred shift and crop, apodisation, scale,
// conj(coil map) and the coil sum; writes (or adds into) the image row.
struct AdjXArgs {
    const float2* in;       // (Z, Y, OSX, ncol)
    int ncol;
    const float2* maps;     // (Z, Y, X, C) or null
    int C, cc, rows;
    int n_img;
    int Z, Y, X, OSX, h, pad;
    const float* apz;
    const float* apy;
    const float* apx;
    float scale;
    const float2* tw;
    FftStages S;
    float2* img;            // (n_img, Z, Y, X)
    int64_t img_stride;
    int accumulate;
    int* err;               // device error word (kDevErr* bits)
    int poll;               // polls before a bounded mbarrier wait gives up
};

__global__ void __launch_bounds__(256) k_adj_x(AdjXArgs a) {
    extern __shared__ float2 sm[];
    const int W = a.rows * a.cc;
    const int L = a.S.L;
    float2* buf0 = sm;
    float2* buf1 = sm + L * W;
    float2* tws = sm + 2 * L * W;
    float2* acc = tws + L;                  // [rows][X]
    for (int i = threadIdx.x; i < L; i += blockDim.x) tws[i] = a.tw[i];
    for (int i = threadIdx.x; i < a.rows * a.X; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);      // images of one row block run side by side
    const int row0 = (int)(blockIdx.x / (unsigned)a.n_img) * a.rows;
    const int nrows = a.Z * a.Y;
    // buffer free during the last stage (the other one is its source)
    float2* ep = (a.S.nstages == 1) ? buf1 : (((a.S.nstages - 1) % 2 == 0) ? buf1 : buf0);
    for (int c0 = 0; c0 < a.C; c0 += a.cc) {
        // stage the [L][W] input tile (centred shift applied on the row index)
        for (int idx = threadIdx.x; idx < L * W; idx += blockDim.x) {
            const int m = idx / W, w = idx - m * W;
            const int rl = w / a.cc, cl = w - rl * a.cc;
            const int row = row0 + rl, c = c0 + cl;
            int j = m + a.h;
            if (j >= L) j -= L;
            int bytes = 0;
            const float2* g = a.in;
            if (row < nrows && c < a.C) {
                bytes = 8;
                g = a.in + ((int64_t)row * a.OSX + j) * a.ncol + (int64_t)img * a.C + c;
            }
            cp_async8(buf0 + idx, g, bytes);
        }
        cp_async_wait_all();
        __syncthreads();
        auto load = [buf0, W](int m, int w) -> float2 { return buf0[m * W + w]; };
        auto store = [&](int k, int w, float2 v) {
            int o = k + a.h - a.pad;
            o %= L;
            if (o < 0) o += L;
            if (o < a.X) ep[o * W + w] = v;
        };
        fft_run(buf0, buf1, tws, a.S, W, true, load, store);
        __syncthreads();
        for (int i = threadIdx.x; i < a.rows * a.X; i += blockDim.x) {
            const int rl = i / a.X, x = i - rl * a.X;
            const int row = row0 + rl;
            if (row >= nrows) continue;
            float2 s = acc[i];
            for (int cl = 0; cl < a.cc && c0 + cl < a.C; ++cl) {
                float2 v = ep[x * W + rl * a.cc + cl];
                if (a.maps) v = cmulc(v, a.maps[((int64_t)row * a.X + x) * a.C + c0 + cl]);
                s = cadd(s, v);
            }
            acc[i] = s;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < a.rows * a.X; i += blockDim.x) {
        const int rl = i / a.X, x = i - rl * a.X;
        const int row = row0 + rl;
        if (row >= nrows) continue;
        const int z = row / a.Y, y = row - z * a.Y;
        const float s = a.apz[z] * a.apy[y] * a.apx[x] * a.scale;
        float2 v = cscale(acc[i], s);
        float2* dst = a.img + (int64_t)img * a.img_stride + (int64_t)row * a.X + x;
        if (a.accumulate) v = cadd(*dst, v);
        *dst = v;
    }
}

// ------------------------------------------------------------------ compile-time variants
// The same three FFT kernels with L and W fixed at compile time (fft_ct):
// used for the transform lengths of the supported workloads.
// Lengths up to 200 use 16-column tiles, longer ones 8-column tiles (the
// shared-memory footprint 2 L W x 8 bytes then allows >= 4 CTAs per SM).
#define TR_CT_WIDE(X) X(60) X(80) X(100) X(120) X(140) X(160) X(200)
#define TR_CT_NARROW(X) X(240) X(320)
#define TR_CT_LENGTHS(X) TR_CT_WIDE(X) TR_CT_NARROW(X)
__host__ __device__ constexpr int ct_width(int L) { return L >= 240 ? 8 : 16; }
// The TMA x passes take 8 coils per CTA at every length: their rows are contiguous,
// so narrow tiles cost no DRAM efficiency and buy occupancy (the strided y / z
// passes keep 16-column tiles up to L = 200: 128-byte row segments).
constexpr int kTmaXWidth = 8;

// Rounds of butterflies an NT-thread CTA runs for the Stockham stages of an
// [L][W] tile.  At L = 320, W = 8 the radix-8 stages have 320 butterflies: 256
// threads need two rounds for them (the second a quarter full), 320 threads one.
__host__ __device__ constexpr int ct_rounds(int L, int W, int NT) {
    int n = 0;
    for (int s = 0; s < ct_nstages(L); ++s) n += ((L / ct_radix(L, s)) * W + NT - 1) / NT;
    return n;
}
// Threads per CTA of the TMA adjoint x pass: 320 for 8-column tiles that then
// take fewer rounds, else 256 (measured on the 160x320x320 grid with 96
// columns: 1 % faster with 320; the forward x pass measured slower with 320 and
// keeps 256).
__host__ __device__ constexpr int ct_threads(int L, int W) {
    return (W <= 8 && ct_rounds(L, W, 320) < ct_rounds(L, W, 256)) ? 320 : 256;
}

// The TMA line passes transform in place (register-held butterflies, one
// [L][W] buffer): half the shared memory of two buffers, so six CTAs of 320
// threads (32 registers each) fit on an SM; 320 threads wherever that takes
// fewer rounds.  Measured 3-5 % faster than the two-buffer transform.
__host__ __device__ constexpr int line_threads(int L, int W) {
    return ct_rounds(L, W, 320) < ct_rounds(L, W, 256) ? 320 : 256;
}
static size_t line_tma_smem_bytes(int L, int W) { return (size_t)(L * W + L) * sizeof(float2) + 128; }
// Threads and CTAs per SM of a line pass with radix plan P (P = 1: two passes,
// one round each: as many threads as the larger pass has butterflies;
// 320 x 8: 128 and 160 -> 160; 160 x 16: 256 and 160 -> 256).
__host__ __device__ constexpr int line_threads_p(int L, int W, int P) {
    return P == 0 ? line_threads(L, W)
                  : ((L / ct_radix_p(P, L, 0)) * W > (L / ct_radix_p(P, L, 1)) * W ? (L / ct_radix_p(P, L, 0)) * W
                                                                                    : (L / ct_radix_p(P, L, 1)) * W);
}
__host__ __device__ constexpr int line_min_ctas(int NT, int P) {
    return P == 0 ? (NT == 320 ? 5 : 6) : (NT <= 160 ? 6 : 4);
}

template <int L, int W, bool INV>
__global__ void __launch_bounds__(256) k_line_ct(LineArgs a) {
    extern __shared__ float2 sm[];
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int64_t q0 = (int64_t)blockIdx.x * W;
    if (lines_unoccupied(a, q0, W)) {
        if (a.skip_zero) lines_write_zeros(a, q0, W, blockIdx.y);
        return;
    }
    const int64_t outer = blockIdx.y;
    const float2* __restrict__ in = a.in + outer * a.Lin * a.inner;
    float2* __restrict__ out = a.out + outer * a.Lout * a.inner;
    for (int i = threadIdx.x; i < L; i += 256) tws[i] = a.tw[i];
    if (a.vec16) {
        constexpr int NCH = W / 2;
#pragma unroll 4
        for (int idx = threadIdx.x; idx < L * NCH; idx += 256) {
            const int m = idx / NCH, ch = idx - m * NCH;
            int j = m + a.h;
            if (j >= L) j -= L;
            const int i = j - a.p_in;
            const int64_t q = q0 + 2 * ch;
            int bytes = 0;
            const float2* g = a.in;
            if (i >= 0 && i < a.Lin && q < a.inner) {
                bytes = (q + 1 < a.inner) ? 16 : 8;
                g = in + (int64_t)i * a.inner + q;
            }
            cp_async16(smA + m * W + 2 * ch, g, bytes);
        }
    } else {
#pragma unroll 4
        for (int idx = threadIdx.x; idx < L * W; idx += 256) {
            const int m = idx / W, w = idx - m * W;
            int j = m + a.h;
            if (j >= L) j -= L;
            const int i = j - a.p_in;
            const int64_t q = q0 + w;
            int bytes = 0;
            const float2* g = a.in;
            if (i >= 0 && i < a.Lin && q < a.inner) {
                bytes = 8;
                g = in + (int64_t)i * a.inner + q;
            }
            cp_async8(smA + idx, g, bytes);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int shift = a.h - a.p_out;
    const int Lout = a.Lout;
    const int64_t inner = a.inner;
    auto store = [&](int k, int w, float2 v) {
        int o = k + shift;
        o = o >= L ? o - L : (o < 0 ? o + L : o);
        const int64_t q = q0 + w;
        if (q < inner && o < Lout) out[(int64_t)o * inner + q] = v;
    };
    fft_ct<L, W, 256, INV>(smA, smB, tws, store);
}

// TMA variant of k_line_ct: the [L][W] tile arrives as two boxes of L/2 rows
// (the centred rotation m -> row (m + L/2) mod L - p_in splits the line in two
// contiguous runs; rows outside [0, Lin) are zero-filled by the TMA unit), the
// transform runs in place in that tile (fft_ct_ip), and two boxes of
// Lout/2 rows leave by TMA stores (rows o = (k + h - p_out) mod L < Lout).
// One thread issues every copy; the rest of the CTA only runs the transform.
// The load wait is bounded: on expiry the CTA waits (bounded) for its copies
// in flight, sets kDevErrTmaWait and exits.
template <int L, int W, bool INV, int P = 0, int NT = line_threads_p(L, W, P)>
__global__ void __launch_bounds__(NT, line_min_ctas(NT, P))
    k_line_tma(LineArgs a, const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout) {
    extern __shared__ __align__(128) unsigned char tsm_raw[];
    __shared__ __align__(8) uint64_t bar;
    // TMA boxes start on 128-byte boundaries (the launch adds 128 bytes of slack)
    float2* tsm = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(tsm_raw) + 127) & ~uintptr_t(127));
    float2* smA = tsm;                               // the [L][W] tile, transformed in place
    float2* tws = tsm + L * W;
    const int q0 = (int)blockIdx.x * W;
    const int outer = (int)blockIdx.y;
    if (lines_unoccupied(a, q0, W)) {                // before any barrier or copy: the CTA leaves whole
        if (a.skip_zero) lines_write_zeros(a, q0, W, blockIdx.y);
        return;
    }
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (unsigned)(L * W * sizeof(float2)));
        tma_load_3d(smA, &tin, &bar, q0, L / 2 - a.p_in, outer);
        tma_load_3d(smA + (L / 2) * W, &tin, &bar, q0, -a.p_in, outer);
    }
    for (int i = threadIdx.x; i < L; i += NT) tws[i] = a.tw[i];
    const bool ok = mbar_wait_or_drain(&bar, 0, a.poll);
    if (__syncthreads_or(!ok)) {          // every thread leaves together
        if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
        return;
    }
    float2* ep = smA;
    auto store = [ep](int k, int w, float2 v) { ep[k * W + w] = v; };
    fft_ct_ip_p<P, L, W, NT, INV>(smA, tws, store);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int half = a.Lout / 2;
        tma_store_3d(&tout, ep + a.kA * W, q0, 0, outer);
        tma_store_3d(&tout, ep + a.kB * W, q0, half, outer);
        tma_store_commit_and_drain();
    }
}

// ------------------------------------------------------------------ fused y + z passes
// The y and z passes of the forward (and the z and y passes of the adjoint)
// in one kernel, so the intermediate (Z, OSY, OSX, ncol) volume never reaches
// HBM.  A thread-block cluster of CL CTAs owns one x column and kYzCW
// k-space columns, i.e. one (z, y) plane of kYzCW columns:
//   forward   CTA r loads the image rows z in [r ZR, r ZR + ZR) of its plane
//             (one 4-D TMA box per half, the y-centring rotation and the zero
//             pad done by the TMA unit as in k_line_tma), transforms them along
//             y in place ([LY][RS] tile, RS = ZR kYzCW), then after a cluster
//             barrier takes the output rows y' in [r YR, r YR + YR): for two y'
//             at a time it gathers the 8 lines' Z inputs from the CTAs holding
//             them (distributed shared memory), transforms along z in place and
//             stores the LZ grid rows by TMA (two boxes: the centring rotation);
//   adjoint   the mirror image: z transforms of its y' rows (TMA loads, two
//             chunks in flight), the Z cropped rows scattered to the CTAs that
//             own them, a cluster barrier, then y transforms of its ZR rows and
//             the Y cropped rows stored by TMA.
// Each line sees exactly the butterflies, twiddles and order of k_line_tma (the
// two-pass plan at 320 points, the default one at 160), so the results equal the
// separate passes bit for bit; plans with TR_PLAN_THREE_PASS_320 do not fuse.  Reads of the plane all
// precede the cluster barrier and writes follow it, so the grid can overwrite
// the x-pass output of the same plane in place (other clusters touch other
// (x, column) planes only).  No TMA multicast: every copy is between global
// memory and the issuing CTA's own shared memory.
// Measured on the 256 x 256 x 128 workload (96 columns, one B200, three-pass y
// transforms in both): 17.5 ms forward and 16.3 ms adjoint, against 7.7 and
// 7.5 ms for the separate passes.
// Each cluster walks its plane as one serial chain (TMA load, y transforms,
// cluster barrier, ten gather / transform / store rounds) at two CTAs per SM,
// so the HBM round trip it saves does not pay; plans run these kernels only
// with TR_PLAN_YZ_FUSION (comparison runs).
constexpr int kYzCW = 4;      // k-space columns per cluster (32-byte rows)
constexpr int kYzNT = 320;    // threads per CTA

struct YzArgs {
    int Z, Y;                 // image lengths along z and y
    int pad_z, pad_y;         // centred zero-pad offsets (L / 2 - n / 2)
    int ncol;
    const float2* twz;        // [LZ] exp(-2 pi i k / LZ)
    const float2* twy;        // [LY]
    int* err;
    int poll;
};

__host__ __device__ constexpr size_t yz_smem_bytes(int LY, int LZ, int ZR) {
    return ((size_t)LY * ZR * kYzCW + 2 * (size_t)LZ * 8 + LY + LZ) * sizeof(float2) + 128;
}

template <int LY, int LZ, int CL, int ZR>
__global__ void __launch_bounds__(kYzNT, 2) k_yz_fwd(YzArgs a, const __grid_constant__ CUtensorMap tin,
                                                    const __grid_constant__ CUtensorMap tout) {
    constexpr int CW = kYzCW, RS = ZR * CW, NT = kYzNT;
    constexpr int YR = ((LY + CL - 1) / CL + 1) / 2 * 2;     // output rows y' per CTA (even)
    static_assert(RS % 16 == 0 && LY % 2 == 0 && LZ % 2 == 0, "fused y/z tile shape");
    extern __shared__ __align__(128) unsigned char yz_raw[];
    __shared__ __align__(8) uint64_t bar;
    float2* ty = align128(yz_raw);          // [LY][RS]: y lines of the CTA's ZR image rows
    float2* tz = ty + LY * RS;              // [2][LZ][8]: z lines of two y' rows (two buffers)
    float2* twy = tz + 2 * LZ * 8;
    float2* twz = twy + LY;
    if (cluster_size() != (unsigned)CL) {  // launched without its cluster: touch no other CTA
        if (threadIdx.x == 0) atomicOr(a.err, kDevErrCluster);
        return;
    }
    const unsigned r = cluster_rank();
    const int cl = (int)(blockIdx.x / (unsigned)CL);
    const int ncg = a.ncol / CW;
    const int x = cl / ncg, c0 = (cl - x * ncg) * CW;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    for (int i = threadIdx.x; i < LY; i += NT) twy[i] = a.twy[i];
    for (int i = threadIdx.x; i < LZ; i += NT) twz[i] = a.twz[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (unsigned)(LY * RS * sizeof(float2)));
        tma_load_4d(ty, &tin, &bar, c0, (int)r * ZR, LY / 2 - a.pad_y, x);
        tma_load_4d(ty + (LY / 2) * RS, &tin, &bar, c0, (int)r * ZR, -a.pad_y, x);
    }
    const bool ok = mbar_wait_or_drain(&bar, 0, a.poll);
    const bool bad = __syncthreads_or(!ok);
    if (bad) {
        if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
    } else {
#pragma unroll 1
        for (int sub = 0; sub < RS / 16; ++sub) {
            float2* b = ty + sub * 16;
            auto store = [b](int k, int w, float2 v) { b[k * RS + w] = v; };
            fft_ct_ip_rs_p<(LY == 320 ? 1 : 0), LY, 16, RS, NT, false>(b, twy, store);
        }
    }
    cluster_sync_all();                     // every y line of the plane is transformed
    const int y_lo = (int)r * YR, y_hi = min(y_lo + YR, LY);
#pragma unroll 1
    for (int i = 0, y0 = y_lo; y0 < y_hi; ++i, y0 += 2) {
        float2* t = tz + (i & 1) * (LZ * 8);
        if (i >= 2) {                       // this buffer's store from two chunks ago has read it
            if (threadIdx.x == 0) tma_store_wait_read<1>();
            __syncthreads();
        }
        // row k of the z line holds image row z = ((k + LZ/2) mod LZ) - pad_z (zero outside [0, Z));
        // column (yl, c) is y' = y0 + yl, k-space column c0 + c
        for (int idx = threadIdx.x; idx < LZ * 4; idx += NT) {
            const int k = idx >> 2, yl = (idx >> 1) & 1, hf = idx & 1;
            int z = k + LZ / 2;
            if (z >= LZ) z -= LZ;
            z -= a.pad_z;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (z >= 0 && z < a.Z) {
                const int q = z / ZR, zl = z - q * ZR;
                int ky = y0 + yl + LY / 2;  // y-transform row of output y' (centring rotation)
                if (ky >= LY) ky -= LY;
                v = dsmem_load4(ty + ky * RS + zl * CW + hf * 2, (unsigned)q);
            }
            reinterpret_cast<float4*>(t)[idx] = v;              // t[k][yl * 4 + hf * 2 .. + 1]
        }
        __syncthreads();
        auto store = [t](int k, int w, float2 v) { t[k * 8 + w] = v; };
        fft_ct_ip<LZ, 8, NT, false>(t, twz, store);
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && !bad) {
            tma_store_4d(&tout, t + (LZ / 2) * 8, c0, y0, 0, x);   // z' in [0, LZ/2): rows [LZ/2, LZ)
            tma_store_4d(&tout, t, c0, y0, LZ / 2, x);             // z' in [LZ/2, LZ): rows [0, LZ/2)
            tma_store_commit();
        }
    }
    if (threadIdx.x == 0) tma_store_wait_read<0>();
    cluster_sync_all();                     // no CTA leaves while another still reads its y tile
}

template <int LY, int LZ, int CL, int ZR>
__global__ void __launch_bounds__(kYzNT, 2) k_yz_adj(YzArgs a, const __grid_constant__ CUtensorMap tin,
                                                    const __grid_constant__ CUtensorMap tout) {
    constexpr int CW = kYzCW, RS = ZR * CW, NT = kYzNT;
    constexpr int YR = ((LY + CL - 1) / CL + 1) / 2 * 2;
    static_assert(RS % 16 == 0 && LY % 2 == 0 && LZ % 2 == 0, "fused y/z tile shape");
    extern __shared__ __align__(128) unsigned char yz_raw[];
    __shared__ __align__(8) uint64_t bar[2];
    float2* ty = align128(yz_raw);          // [LY][RS]: y lines of the CTA's ZR output rows
    float2* tz = ty + LY * RS;              // [2][LZ][8]
    float2* twy = tz + 2 * LZ * 8;
    float2* twz = twy + LY;
    if (cluster_size() != (unsigned)CL) {  // launched without its cluster: touch no other CTA
        if (threadIdx.x == 0) atomicOr(a.err, kDevErrCluster);
        return;
    }
    const unsigned r = cluster_rank();
    const int cl = (int)(blockIdx.x / (unsigned)CL);
    const int ncg = a.ncol / CW;
    const int x = cl / ncg, c0 = (cl - x * ncg) * CW;
    const int y_lo = (int)r * YR, y_hi = min(y_lo + YR, LY);
    const int nchunk = y_hi > y_lo ? (y_hi - y_lo) / 2 : 0;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    for (int i = threadIdx.x; i < LY; i += NT) twy[i] = a.twy[i];
    for (int i = threadIdx.x; i < LZ; i += NT) twz[i] = a.twz[i];
    __syncthreads();
    // grid rows z' of two y' rows: transform row k holds z' = (k + LZ/2) mod LZ
    auto issue = [&](int i) {
        float2* t = tz + (i & 1) * (LZ * 8);
        mbar_expect_tx(&bar[i & 1], (unsigned)(LZ * 8 * sizeof(float2)));
        tma_load_4d(t, &tin, &bar[i & 1], c0, y_lo + 2 * i, LZ / 2, x);
        tma_load_4d(t + (LZ / 2) * 8, &tin, &bar[i & 1], c0, y_lo + 2 * i, 0, x);
    };
    if (threadIdx.x == 0) {
        if (nchunk > 0) issue(0);
        if (nchunk > 1) issue(1);
    }
    bool bad = false;
#pragma unroll 1
    for (int i = 0; i < nchunk; ++i) {
        float2* t = tz + (i & 1) * (LZ * 8);
        const bool ok = mbar_wait_or_drain(&bar[i & 1], (unsigned)((i >> 1) & 1), a.poll);
        if (__syncthreads_or(!ok)) {
            // the other buffer's copy may be in flight: let it land, then stop loading
            if (i + 1 < nchunk)
                mbar_wait_bounded(&bar[(i + 1) & 1], (unsigned)(((i + 1) >> 1) & 1), kMbarDrainLimit);
            if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
            bad = true;
            break;
        }
        auto store = [t](int k, int w, float2 v) { t[k * 8 + w] = v; };
        fft_ct_ip<LZ, 8, NT, true>(t, twz, store);
        __syncthreads();
        // output row z (cropped) is transform row (z - Z/2) mod LZ; it belongs to CTA z / ZR, whose
        // y-transform row for y' = y_lo + 2 i + yl is (y' + LY/2) mod LY
        for (int idx = threadIdx.x; idx < a.Z * 4; idx += NT) {
            const int z = idx >> 2, yl = (idx >> 1) & 1, hf = idx & 1;
            int kz = z - a.Z / 2;
            if (kz < 0) kz += LZ;
            const float4 v = reinterpret_cast<const float4*>(t)[kz * 4 + yl * 2 + hf];
            const int q = z / ZR, zl = z - q * ZR;
            int ky = y_lo + 2 * i + yl + LY / 2;
            if (ky >= LY) ky -= LY;
            dsmem_store4(ty + ky * RS + zl * CW + hf * 2, (unsigned)q, v);
        }
        fence_proxy_async_smem();           // generic reads of t before the next TMA write into it
        __syncthreads();
        if (threadIdx.x == 0 && i + 2 < nchunk) issue(i + 2);
    }
    cluster_sync_all();                     // every z-transformed row has reached its owner
    if (!bad) {
#pragma unroll 1
        for (int sub = 0; sub < RS / 16; ++sub) {
            float2* b = ty + sub * 16;
            auto store = [b](int k, int w, float2 v) { b[k * RS + w] = v; };
            fft_ct_ip_rs_p<(LY == 320 ? 1 : 0), LY, 16, RS, NT, true>(b, twy, store);
        }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0 && !bad) {
        // output y in [0, Y/2): transform rows [LY - Y/2, LY); y in [Y/2, Y): rows [0, Y/2)
        tma_store_4d(&tout, ty + (LY - a.Y / 2) * RS, c0, (int)r * ZR, 0, x);
        tma_store_4d(&tout, ty, c0, (int)r * ZR, a.Y / 2, x);
        tma_store_commit_and_drain();
    }
}

template <int L, int W>
__global__ void __launch_bounds__(256) k_fwd_x_ct(FwdXArgs a) {
    extern __shared__ float2 sm[];
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);      // images of one row block run side by side
    const int row0 = (int)(blockIdx.x / (unsigned)a.n_img) * a.rows;
    const int c0 = blockIdx.z * a.cc;
    const int nrows = a.Z * a.Y;
    const int cc = a.cc;
    const float2* __restrict__ src = a.img + (int64_t)img * a.img_stride;
    for (int i = threadIdx.x; i < L; i += 256) tws[i] = a.tw[i];
#pragma unroll 4
    for (int idx = threadIdx.x; idx < L * W; idx += 256) {
        const int m = idx / W, w = idx - m * W;
        const int rl = w / cc, cl = w - rl * cc;
        const int row = row0 + rl, c = c0 + cl;
        int j = m + a.h;
        if (j >= L) j -= L;
        const int x = j - a.pad;
        float2 v = make_float2(0.f, 0.f);
        if (x >= 0 && x < a.X && row < nrows && c < a.C) {
            const int z = row / a.Y, y = row - z * a.Y;
            v = src[(int64_t)row * a.X + x];
            if (a.maps) v = cmul(v, a.maps[((int64_t)row * a.X + x) * a.C + c]);
            v = cscale(v, a.apz[z] * a.apy[y] * a.apx[x] * a.scale);
        }
        smA[idx] = v;
    }
    __syncthreads();
    const int h = a.h;
    auto store = [&](int k, int w, float2 v) {
        const int rl = w / cc, cl = w - rl * cc;
        const int row = row0 + rl, c = c0 + cl;
        if (row >= nrows || c >= a.C) return;
        int g = k + h;
        if (g >= L) g -= L;
        a.out[((int64_t)row * a.OSX + g) * a.ncol + (int64_t)img * a.C + c] = v;
    };
    fft_ct<L, W, 256, false>(smA, smB, tws, store);
}

template <int L, int W>
__global__ void __launch_bounds__(256) k_adj_x_ct(AdjXArgs a) {
    extern __shared__ float2 sm[];
    float2* buf0 = sm;
    float2* buf1 = sm + L * W;
    float2* tws = sm + 2 * L * W;
    float2* acc = tws + L;                  // [rows][X]
    for (int i = threadIdx.x; i < L; i += 256) tws[i] = a.tw[i];
    for (int i = threadIdx.x; i < a.rows * a.X; i += 256) acc[i] = make_float2(0.f, 0.f);
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);      // images of one row block run side by side
    const int row0 = (int)(blockIdx.x / (unsigned)a.n_img) * a.rows;
    const int nrows = a.Z * a.Y;
    const int cc = a.cc;
    float2* ep = fft_ct_free<L>(buf0, buf1);
    const int shift = a.h - a.pad;
    for (int c0 = 0; c0 < a.C; c0 += cc) {
#pragma unroll 4
        for (int idx = threadIdx.x; idx < L * W; idx += 256) {
            const int m = idx / W, w = idx - m * W;
            const int rl = w / cc, cl = w - rl * cc;
            const int row = row0 + rl, c = c0 + cl;
            int j = m + a.h;
            if (j >= L) j -= L;
            int bytes = 0;
            const float2* g = a.in;
            if (row < nrows && c < a.C) {
                bytes = 8;
                g = a.in + ((int64_t)row * a.OSX + j) * a.ncol + (int64_t)img * a.C + c;
            }
            cp_async8(buf0 + idx, g, bytes);
        }
        cp_async_wait_all();
        __syncthreads();
        const int X = a.X;
        auto store = [&](int k, int w, float2 v) {
            int o = k + shift;
            o = o >= L ? o - L : (o < 0 ? o + L : o);
            if (o < X) ep[o * W + w] = v;
        };
        fft_ct<L, W, 256, true>(buf0, buf1, tws, store);
        __syncthreads();
        for (int i = threadIdx.x; i < a.rows * X; i += 256) {
            const int rl = i / X, x = i - rl * X;
            const int row = row0 + rl;
            if (row >= nrows) continue;
            float2 s = acc[i];
            for (int cl = 0; cl < cc && c0 + cl < a.C; ++cl) {
                float2 v = ep[x * W + rl * cc + cl];
                if (a.maps) v = cmulc(v, a.maps[((int64_t)row * X + x) * a.C + c0 + cl]);
                s = cadd(s, v);
            }
            acc[i] = s;
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < a.rows * a.X; i += 256) {
        const int rl = i / a.X, x = i - rl * a.X;
        const int row = row0 + rl;
        if (row >= nrows) continue;
        const int z = row / a.Y, y = row - z * a.Y;
        const float sc = a.apz[z] * a.apy[y] * a.apx[x] * a.scale;
        float2 v = cscale(acc[i], sc);
        float2* dst = a.img + (int64_t)img * a.img_stride + (int64_t)row * a.X + x;
        if (a.accumulate) v = cadd(*dst, v);
        *dst = v;
    }
}

// ------------------------------------------------------------------ staged x-pass variants
// W = 16 columns = ROWS image rows x CC coils (CC in {4, 8, 16}).  Forward:
// each row's image values and its contiguous coil-map row are staged in shared
// memory with cp.async, the products formed there.  Adjoint: the coil
// combination runs with one thread per (x, coil) and a shuffle reduction over
// the CC lanes of a coil group (no bank conflicts).
template <int L, int W, int CC>
__global__ void __launch_bounds__(256) k_fwd_x_st(FwdXArgs a) {
    constexpr int ROWS = W / CC;
    extern __shared__ float2 sm[];
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int X = a.X;
    float2* s_img = smB;                 // [ROWS][X]
    float2* s_map = smB + ROWS * X;      // [ROWS][X][CC]
    __shared__ float s_apzy[ROWS];
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);      // images of one row block run side by side
    const int row0 = (int)(blockIdx.x / (unsigned)a.n_img) * ROWS;
    const int c0 = blockIdx.z * CC;
    const int nrows = a.Z * a.Y;
    const float2* __restrict__ src = a.img + (int64_t)img * a.img_stride;
    for (int i = threadIdx.x; i < L; i += 256) tws[i] = a.tw[i];
    if (threadIdx.x < ROWS) {
        const int row = row0 + threadIdx.x;
        float v = 0.f;
        if (row < nrows) {
            const int z = row / a.Y, y = row - z * a.Y;
            v = a.apz[z] * a.apy[y] * a.scale;
        }
        s_apzy[threadIdx.x] = v;
    }
    for (int i = threadIdx.x; i < ROWS * X; i += 256) {
        const int rl = i / X, x = i - rl * X;
        const int row = row0 + rl;
        cp_async8(s_img + i, row < nrows ? src + (int64_t)row * X + x : src, row < nrows ? 8 : 0);
    }
    if (a.maps) {
        for (int i = threadIdx.x; i < ROWS * X * CC; i += 256) {
            const int rl = i / (X * CC), rem = i - rl * X * CC;
            const int x = rem / CC, cl = rem - x * CC;
            const int row = row0 + rl, c = c0 + cl;
            const bool ok = row < nrows && c < a.C;
            cp_async8(s_map + i, ok ? a.maps + ((int64_t)row * X + x) * a.C + c : a.maps, ok ? 8 : 0);
        }
    }
    cp_async_wait_all();
    __syncthreads();
#pragma unroll 4
    for (int idx = threadIdx.x; idx < L * W; idx += 256) {
        const int m = idx / W, w = idx - m * W;
        const int rl = w / CC, cl = w - rl * CC;
        int j = m + a.h;
        if (j >= L) j -= L;
        const int x = j - a.pad;
        float2 v = make_float2(0.f, 0.f);
        if (x >= 0 && x < X) {
            v = s_img[rl * X + x];
            if (a.maps) v = cmul(v, s_map[(rl * X + x) * CC + cl]);
            v = cscale(v, s_apzy[rl] * a.apx[x]);
        }
        smA[idx] = v;
    }
    __syncthreads();
    const int h = a.h;
    auto store = [&](int k, int w, float2 v) {
        const int rl = w / CC, cl = w - rl * CC;
        const int row = row0 + rl, c = c0 + cl;
        if (row >= nrows || c >= a.C) return;
        int g = k + h;
        if (g >= L) g -= L;
        a.out[((int64_t)row * a.OSX + g) * a.ncol + (int64_t)img * a.C + c] = v;
    };
    fft_ct<L, W, 256, false>(smA, smB, tws, store);
}

template <int L, int W, int CC>
__global__ void __launch_bounds__(256) k_adj_x_st(AdjXArgs a) {
    constexpr int ROWS = W / CC;
    extern __shared__ float2 sm[];
    float2* buf0 = sm;
    float2* buf1 = sm + L * W;
    float2* tws = sm + 2 * L * W;
    float2* acc = tws + L;                  // [ROWS][X]
    for (int i = threadIdx.x; i < L; i += 256) tws[i] = a.tw[i];
    for (int i = threadIdx.x; i < ROWS * a.X; i += 256) acc[i] = make_float2(0.f, 0.f);
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);      // images of one row block run side by side
    const int row0 = (int)(blockIdx.x / (unsigned)a.n_img) * ROWS;
    const int nrows = a.Z * a.Y;
    const int X = a.X;
    float2* ep = fft_ct_free<L>(buf0, buf1);
    const int shift = a.h - a.pad;
    for (int c0 = 0; c0 < a.C; c0 += CC) {
#pragma unroll 4
        for (int idx = threadIdx.x; idx < L * W; idx += 256) {
            const int m = idx / W, w = idx - m * W;
            const int rl = w / CC, cl = w - rl * CC;
            const int row = row0 + rl, c = c0 + cl;
            int j = m + a.h;
            if (j >= L) j -= L;
            const bool ok = row < nrows && c < a.C;
            cp_async8(buf0 + idx, ok ? a.in + ((int64_t)row * a.OSX + j) * a.ncol + (int64_t)img * a.C + c : a.in,
                      ok ? 8 : 0);
        }
        cp_async_wait_all();
        __syncthreads();
        auto store = [&](int k, int w, float2 v) {
            int o = k + shift;
            o = o >= L ? o - L : (o < 0 ? o + L : o);
            if (o < X) ep[o * W + w] = v;
        };
        fft_ct<L, W, 256, true>(buf0, buf1, tws, store);
        __syncthreads();
        // thread (x, w): conj(S) product, then a sum over the CC lanes of one row.
        // Every lane runs every iteration (the shuffles need the whole warp).
        for (int base = 0; base < X * W; base += 256) {
            const int i = base + (int)threadIdx.x;
            const bool live = i < X * W;
            const int x = i / W, w = i - x * W;
            const int rl = w / CC, cl = w - rl * CC;
            const int row = row0 + rl, c = c0 + cl;
            float2 v = make_float2(0.f, 0.f);
            if (live && row < nrows && c < a.C) {
                v = ep[i];
                if (a.maps) v = cmulc(v, a.maps[((int64_t)row * X + x) * a.C + c]);
            }
#pragma unroll
            for (int o = CC / 2; o > 0; o >>= 1) {
                v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
                v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
            }
            if (live && cl == 0) acc[rl * X + x] = cadd(acc[rl * X + x], v);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < ROWS * X; i += 256) {
        const int rl = i / X, x = i - rl * X;
        const int row = row0 + rl;
        if (row >= nrows) continue;
        const int z = row / a.Y, y = row - z * a.Y;
        const float sc = a.apz[z] * a.apy[y] * a.apx[x] * a.scale;
        float2 v = cscale(acc[i], sc);
        float2* dst = a.img + (int64_t)img * a.img_stride + (int64_t)row * X + x;
        if (a.accumulate) v = cadd(*dst, v);
        *dst = v;
    }
}

// ------------------------------------------------------------------ TMA x-pass variants
// One image row x W coils per CTA (W = CC).  Forward: the image row and the
// row's W coil-map columns arrive by TMA in the FFT's second buffer, the
// product (apodisation, scale, centred zero-pad) fills the first, and the
// transformed [L][W] tile leaves as two TMA boxes of L/2 rows (the centred
// shift g = (k + L/2) mod L splits it in two).  Adjoint: per coil group the
// [L][W] tile arrives as two boxes (rows rotated by L/2), the inverse FFT
// writes the cropped row into shared memory, and the conj(S) product and the
// coil sum run as in k_adj_x_st.  Loads complete on one mbarrier (phase per
// coil group) with a bounded wait.

template <int L, int W, int NT = 256>
__global__ void __launch_bounds__(NT) k_fwd_x_tma(FwdXArgs a, const __grid_constant__ CUtensorMap timg,
                                                   const __grid_constant__ CUtensorMap tmap,
                                                   const __grid_constant__ CUtensorMap tout) {
    extern __shared__ __align__(128) unsigned char xsm_raw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ float s_apzy;
    float2* sm = align128(xsm_raw);
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int X = a.X;
    float2* s_img = smA;              // [X]     (the first FFT stage reads these and writes smB)
    float2* s_map = smA + X;          // [X][W]
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);
    const int row = (int)(blockIdx.x / (unsigned)a.n_img);
    const int c0 = (int)blockIdx.z * W;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (unsigned)(X * (W + 1) * sizeof(float2)));
        tma_load_3d(s_img, &timg, &bar, 0, row, img);
        tma_load_3d(s_map, &tmap, &bar, c0, 0, row);
        const int z = row / a.Y, y = row - z * a.Y;
        s_apzy = a.apz[z] * a.apy[y] * a.scale;
    }
    for (int i = threadIdx.x; i < L; i += NT) tws[i] = a.tw[i];
    const bool ok = mbar_wait_or_drain(&bar, 0, a.poll);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
        return;
    }
    const float apzy = s_apzy;
    const int h = a.h, pad = a.pad;
    const float* apx = a.apx;
    // input element m of column w: u * S * apodisation * scale at x = (m + L/2) mod L - pad, 0 outside the
    // image (scaling the image row once in shared memory first measured 1 % slower: one more barrier)
    auto load = [=](int m, int w) {
        int j = m + h;
        if (j >= L) j -= L;
        const int x = j - pad;
        float2 v = make_float2(0.f, 0.f);
        if (x >= 0 && x < X) v = cscale(cmul(s_img[x], s_map[x * W + w]), apzy * apx[x]);
        return v;
    };
    float2* ep = fft_ct_free<L>(smA, smB);
    auto store = [ep](int k, int w, float2 v) { ep[k * W + w] = v; };
    fft_ct_ld<L, W, NT, false>(smA, smB, tws, load, store);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int col = img * a.C + c0;
        tma_store_3d(&tout, ep + (L / 2) * W, col, 0, row);
        tma_store_3d(&tout, ep, col, L / 2, row);
        tma_store_commit_and_drain();
    }
}

// PF: the coil maps of each group are loaded into registers before the
// transform (in flight during it); otherwise in the epilogue.  MINB: CTAs per
// SM the register allocation is sized for.  At L = 320, W = 8 the epilogue
// loads with four CTAs per SM (48 registers) measured 4 % faster than the
// prefetch with three (64 registers); the prefetch with four spills.
template <int L, int W, int NT = ct_threads(L, W), bool PF = false, int MINB = 4>
__global__ void __launch_bounds__(NT, MINB) k_adj_x_tma(AdjXArgs a, const __grid_constant__ CUtensorMap tin) {
    extern __shared__ __align__(128) unsigned char xsm_raw[];
    __shared__ __align__(8) uint64_t bar;
    float2* sm = align128(xsm_raw);
    float2* buf0 = sm;
    float2* buf1 = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int X = a.X;                      // <= 256 <= NT: thread x owns image column x
    const int XP = X + 4;                   // padded row of the [W][XP] epilogue tile
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);
    const int row = (int)(blockIdx.x / (unsigned)a.n_img);
    const int x = threadIdx.x;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    for (int i = threadIdx.x; i < L; i += NT) tws[i] = a.tw[i];
    float2* ep = fft_ct_free<L>(buf0, buf1);
    const int shift = a.h - a.pad;
    const float4* mrow = reinterpret_cast<const float4*>(a.maps + ((int64_t)row * X + x) * a.C);
    float2 s = make_float2(0.f, 0.f);
    // the transform's last stage does not read buf0 when it writes buf1 (odd stage
    // counts): the next group's tile then loads during this group's epilogue
    constexpr bool kEarly = (ct_nstages(L) % 2) == 1;
    auto issue = [&](int c0) {
        mbar_expect_tx(&bar, (unsigned)(L * W * sizeof(float2)));
        const int col = img * a.C + c0;
        tma_load_3d(buf0, &tin, &bar, col, L / 2, row);
        tma_load_3d(buf0 + (L / 2) * W, &tin, &bar, col, 0, row);
    };
    __syncthreads();                        // barrier initialised
    if (threadIdx.x == 0) issue(0);
    int phase = 0;
    for (int c0 = 0; c0 < a.C; c0 += W, phase ^= 1) {
        // this column's W coil-map values, in flight during the transform (PF)
        float4 m2[W / 2];
        if (PF && x < X) {
#pragma unroll
            for (int q = 0; q < W / 2; ++q) m2[q] = mrow[(c0 >> 1) + q];
        }
        const bool ok = mbar_wait_or_drain(&bar, (unsigned)phase, a.poll);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
            return;
        }
        auto store = [&](int k, int w, float2 v) {
            int o = k + shift;
            o = o >= L ? o - L : (o < 0 ? o + L : o);
            if (o < X) ep[w * XP + o] = v;
        };
        fft_ct<L, W, NT, true>(buf0, buf1, tws, store);
        __syncthreads();                    // transform done: buf0 free (odd stage counts), ep complete
        if (kEarly && threadIdx.x == 0 && c0 + W < a.C) issue(c0 + W);
        // conj(S) product and the sum over this group's coils, in coil order
        if (x < X) {
            if (!PF) {
#pragma unroll
                for (int q = 0; q < W / 2; ++q) m2[q] = mrow[(c0 >> 1) + q];
            }
#pragma unroll
            for (int q = 0; q < W / 2; ++q) {
                s = cadd(s, cmulc(ep[(2 * q) * XP + x], make_float2(m2[q].x, m2[q].y)));
                s = cadd(s, cmulc(ep[(2 * q + 1) * XP + x], make_float2(m2[q].z, m2[q].w)));
            }
        }
        if (!kEarly) {
            __syncthreads();                // the epilogue's reads of ep (= buf0) are done
            if (threadIdx.x == 0 && c0 + W < a.C) issue(c0 + W);
        }
    }
    if (x < X) {
        const int z = row / a.Y, y = row - z * a.Y;
        float2 v = cscale(s, a.apz[z] * a.apy[y] * a.scale * a.apx[x]);
        float2* dst = a.img + (int64_t)img * a.img_stride + (int64_t)row * X + x;
        if (a.accumulate) v = cadd(*dst, v);
        *dst = v;
    }
}

// ------------------------------------------------------------------ two-pass TMA x passes
// The same work as k_fwd_x_tma / k_adj_x_tma with the L-point transform in two
// passes through shared memory (radix plan 1: 320 = 20 x 16) instead of three
// (5, 8, 8).  The x passes are bound by the shared-memory data pipe (ncu on
// k_adj_x_tma: LSU wavefronts at 88 % of peak, DRAM at 40 %), and a pass
// moves every element through shared memory once each way.  kWideNT threads:
// the radix-16 pass has L/16 x W = 160 butterflies, the radix-20 pass 128.
constexpr int kWideNT = 160;

template <int L, int W>
__global__ void __launch_bounds__(kWideNT, 5) k_fwd_x_wide(FwdXArgs a, const __grid_constant__ CUtensorMap timg,
                                                           const __grid_constant__ CUtensorMap tmap,
                                                           const __grid_constant__ CUtensorMap tout) {
    constexpr int NT = kWideNT;
    extern __shared__ __align__(128) unsigned char xsm_raw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ float s_apzy;
    float2* sm = align128(xsm_raw);
    float2* smA = sm;
    float2* smB = sm + L * W;
    float2* tws = sm + 2 * L * W;
    const int X = a.X;
    float2* s_img = smA;              // [X]     (the first pass reads these and writes smB)
    float2* s_map = smA + X;          // [X][W]
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);
    const int row = (int)(blockIdx.x / (unsigned)a.n_img);
    const int c0 = (int)blockIdx.z * W;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(&bar, (unsigned)(X * (W + 1) * sizeof(float2)));
        tma_load_3d(s_img, &timg, &bar, 0, row, img);
        tma_load_3d(s_map, &tmap, &bar, c0, 0, row);
        const int z = row / a.Y, y = row - z * a.Y;
        s_apzy = a.apz[z] * a.apy[y] * a.scale;
    }
    for (int i = threadIdx.x; i < L; i += NT) tws[i] = a.tw[i];
    const bool ok = mbar_wait_or_drain(&bar, 0, a.poll);
    if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
        return;
    }
    const float apzy = s_apzy;
    const int h = a.h, pad = a.pad;
    const float* apx = a.apx;
    auto load = [=](int m, int w) {
        int j = m + h;
        if (j >= L) j -= L;
        const int x = j - pad;
        float2 v = make_float2(0.f, 0.f);
        if (x >= 0 && x < X) v = cscale(cmul(s_img[x], s_map[x * W + w]), apzy * apx[x]);
        return v;
    };
    float2* ep = fft_ct_free<L, 1>(smA, smB);        // smA: the staged row is read by the first pass only
    auto store = [ep](int k, int w, float2 v) { ep[k * W + w] = v; };
    fft_ct_ld_p<1, L, W, NT, false>(smA, smB, tws, load, store);
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int col = img * a.C + c0;
        tma_store_3d(&tout, ep + (L / 2) * W, col, 0, row);
        tma_store_3d(&tout, ep, col, L / 2, row);
        tma_store_commit_and_drain();
    }
}

// Adjoint: the coil groups' tiles alternate between the two buffers, so the
// next group's tile loads into the buffer the second pass has just read while
// this group's epilogue reads the cropped rows written over its input tile.
// Epilogue: lane l of a warp takes image column x = 16 b + l / 2 of block b
// (blocks dealt to the warps in turn) and coils 4 (l % 2) .. 4 (l % 2) + 3 of
// the group, so a warp's coil-map loads cover 1 KB in 8 (C = 8) or 16 lines
// instead of one 64-byte piece per thread in 32.  The two lanes of a column
// exchange one component each (one shuffle): the even lane forms the real part
// of the group's sum, the odd lane the imaginary part, and each adds its scaled
// float into the image row (the first group writes it; a warp's stores are 128
// contiguous bytes, and the row stays in L2 between the groups).  Holding the
// sums in registers across the transforms instead spilled and measured 4 %
// slower (3.23 against 3.10 ms on the 96-column bench bin).
constexpr int kWideXBlocks = 4;               // ceil(256 / 16 / (kWideNT / 32)): X <= 256

template <int L, int W>
__global__ void __launch_bounds__(kWideNT, 5) k_adj_x_wide(AdjXArgs a, const __grid_constant__ CUtensorMap tin) {
    constexpr int NT = kWideNT;
    constexpr int NW = NT / 32;
    static_assert(W == 8, "four coils per lane of a 2-lane column group");
    extern __shared__ __align__(128) unsigned char xsm_raw[];
    __shared__ __align__(8) uint64_t bar;
    float2* sm = align128(xsm_raw);
    float2* tin_buf = sm;                   // this group's input tile; the epilogue rows after pass 1
    float2* work = sm + L * W;              // pass-1 output; the next group's input tile
    float2* tws = sm + 2 * L * W;
    const int X = a.X;
    // [W][XP] epilogue tile; XP = 2 mod 16 puts the second pass's stores of the
    // 8 columns of one output row in 8 different 4-bank groups
    const int XP = X + 2;
    const int img = (int)(blockIdx.x % (unsigned)a.n_img);
    const int row = (int)(blockIdx.x / (unsigned)a.n_img);
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5;
    const int hf = lane & 1;                // coils 4 hf .. 4 hf + 3 of the group
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    for (int i = threadIdx.x; i < L; i += NT) tws[i] = a.tw[i];
    const int shift = a.h - a.pad;
    const float4* mrow = reinterpret_cast<const float4*>(a.maps + (int64_t)row * X * a.C);
    const int z = row / a.Y, y = row - z * a.Y;
    const float szy = a.apz[z] * a.apy[y] * a.scale;
    auto issue = [&](int c0, float2* dst) {
        mbar_expect_tx(&bar, (unsigned)(L * W * sizeof(float2)));
        const int col = img * a.C + c0;
        tma_load_3d(dst, &tin, &bar, col, L / 2, row);
        tma_load_3d(dst + (L / 2) * W, &tin, &bar, col, 0, row);
    };
    __syncthreads();                        // barrier initialised
    if (threadIdx.x == 0) issue(0, tin_buf);
    int phase = 0;
    for (int c0 = 0; c0 < a.C; c0 += W, phase ^= 1) {
        // one thread polls; the CTA barrier after it is also the barrier between
        // the previous epilogue's reads and this group's first pass
        const bool ok = threadIdx.x == 0 ? mbar_wait_or_drain(&bar, (unsigned)phase, a.poll) : true;
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicOr(a.err, kDevErrTmaWait);
            return;
        }
        float2* ep = tin_buf;
        auto store = [&](int k, int w, float2 v) {
            int o = k + shift;
            o = o >= L ? o - L : (o < 0 ? o + L : o);
            if (o < X) ep[w * XP + o] = v;
        };
        fft_ct_p<1, L, W, NT, true>(tin_buf, work, tws, store);
        __syncthreads();                    // pass 2 done: `work` free, ep complete
        if (threadIdx.x == 0 && c0 + W < a.C) issue(c0 + W, work);
        // conj(S) product and the sum over this group's coils
#pragma unroll
        for (int b = 0; b < kWideXBlocks; ++b) {
            const int x = 16 * (warp + NW * b) + (lane >> 1);
            if (16 * (warp + NW * b) < X) {             // whole blocks: X % 16 == 0
                const float4* mp = mrow + ((int64_t)x * a.C + c0) / 2 + 2 * hf;
                const float4 m0 = mp[0], m1 = mp[1];
                const float2* e = ep + (4 * hf) * XP + x;
                float2 t = cmulc(e[0], make_float2(m0.x, m0.y));
                t = cadd(t, cmulc(e[XP], make_float2(m0.z, m0.w)));
                t = cadd(t, cmulc(e[2 * XP], make_float2(m1.x, m1.y)));
                t = cadd(t, cmulc(e[3 * XP], make_float2(m1.z, m1.w)));
                // lane 2i forms t0.x + t1.x, lane 2i + 1 t0.y + t1.y; each adds its
                // scaled float into the image row (the first group writes it)
                const float recv = __shfl_xor_sync(0xffffffffu, hf ? t.x : t.y, 1);
                float v = (hf ? recv + t.y : t.x + recv) * (szy * a.apx[x]);
                float* dst = reinterpret_cast<float*>(a.img + (int64_t)img * a.img_stride + (int64_t)row * X + x) + hf;
                if (a.accumulate || c0 > 0) v = *dst + v;
                *dst = v;
            }
        }
        float2* t = tin_buf;
        tin_buf = work;
        work = t;
    }
}

// ------------------------------------------------------------------ per-sample tap records
// First tap per axis and the 15 KB weights of every (sorted) sample, computed
// once at plan creation; interpolation and gridding read them instead of
// re-evaluating the window.  w[0..4] z taps, w[5..9] y taps, w[10..14] x taps.
struct __align__(16) TapRec {
    int4 b;          // (bz, by, bx, 0): first tap on the oversampled grid (may be < 0)
    float4 w[4];
};

__global__ void k_prep_taps(const float4* __restrict__ ks, int64_t M, float beta, TapRec* __restrict__ out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= M) return;
    const float4 k = ks[s];
    float wz[5], wy[5], wx[5];
    const int bz = axis_taps(k.x, beta, wz);
    const int by = axis_taps(k.y, beta, wy);
    const int bx = axis_taps(k.z, beta, wx);
    TapRec r;
    r.b = make_int4(bz, by, bx, 0);
    r.w[0] = make_float4(wz[0], wz[1], wz[2], wz[3]);
    r.w[1] = make_float4(wz[4], wy[0], wy[1], wy[2]);
    r.w[2] = make_float4(wy[3], wy[4], wx[0], wx[1]);
    r.w[3] = make_float4(wx[2], wx[3], wx[4], 0.f);
    out[s] = r;
}

// ------------------------------------------------------------------ interpolation
// G lanes cooperate on one sample (lane = column group); taps read ncol
// contiguous complex values per grid point (coalesced across lanes).
template <int CPL>
__global__ void __launch_bounds__(256) k_interp(const float2* __restrict__ grid, const TapRec* __restrict__ taps,
                                                int64_t M, int ncol, int G, int os0, int os1, int os2,
                                                int mode, float sigma, const float2* __restrict__ y,
                                                float2* __restrict__ out) {
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t s = gt / G;
    const int lane = (int)(gt - s * G);
    if (s >= M) return;
    const TapRec rec = taps[s];
    const float wz[5] = {rec.w[0].x, rec.w[0].y, rec.w[0].z, rec.w[0].w, rec.w[1].x};
    const float wy[5] = {rec.w[1].y, rec.w[1].z, rec.w[1].w, rec.w[2].x, rec.w[2].y};
    const float wx[5] = {rec.w[2].z, rec.w[2].w, rec.w[3].x, rec.w[3].y, rec.w[3].z};
    const int bz = rec.b.x, by = rec.b.y, bx = rec.b.z;
    int iy[5], ix[5];
#pragma unroll
    for (int t = 0; t < 5; ++t) {
        iy[t] = pmod(by + t, os1);
        ix[t] = pmod(bx + t, os2);
    }
    float2 acc[CPL];
#pragma unroll
    for (int j = 0; j < CPL; ++j) acc[j] = make_float2(0.f, 0.f);
    if (wz[4] == 0.f && wy[4] == 0.f && wx[4] == 0.f) {
        // common case: four taps per axis (k - 2 not an integer), fully unrolled
#pragma unroll
        for (int tz = 0; tz < 4; ++tz) {
            const int64_t zoff = (int64_t)pmod(bz + tz, os0) * os1;
#pragma unroll
            for (int ty = 0; ty < 4; ++ty) {
                const float wzy = wz[tz] * wy[ty];
                const int64_t yoff = (zoff + iy[ty]) * os2;
#pragma unroll
                for (int tx = 0; tx < 4; ++tx) {
                    const float w = wzy * wx[tx];
                    const float2* gp = grid + (yoff + ix[tx]) * ncol;
#pragma unroll
                    for (int j = 0; j < CPL; ++j) {
                        const int col = lane + j * G;
                        if (col < ncol) {
                            acc[j] = cfma_real(w, gp[col], acc[j]);
                        }
                    }
                }
            }
        }
    } else
#pragma unroll 1
    for (int tz = 0; tz < 5; ++tz) {
        if (wz[tz] == 0.f) continue;
        const int64_t zoff = (int64_t)pmod(bz + tz, os0) * os1;
#pragma unroll
        for (int ty = 0; ty < 5; ++ty) {
            if (wy[ty] == 0.f) continue;
            const float wzy = wz[tz] * wy[ty];
            const int64_t yoff = (zoff + iy[ty]) * os2;
#pragma unroll
            for (int tx = 0; tx < 5; ++tx) {
                if (wx[tx] == 0.f) continue;
                const float w = wzy * wx[tx];
                const float2* gp = grid + (yoff + ix[tx]) * ncol;
#pragma unroll
                for (int j = 0; j < CPL; ++j) {
                    const int col = lane + j * G;
                    if (col < ncol) {
                        acc[j] = cfma_real(w, gp[col], acc[j]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int j = 0; j < CPL; ++j) {
        const int col = lane + j * G;
        if (col >= ncol) continue;
        const int64_t o = s * ncol + col;
        if (mode == kInterpDualProx) {
            const float2 r = csub(acc[j], y[o]);
            const float2 q = out[o];
            const float inv = 1.0f / (1.0f + sigma);
            out[o] = make_float2((q.x + sigma * r.x) * inv, (q.y + sigma * r.y) * inv);
        } else {
            out[o] = acc[j];
        }
    }
}

// ------------------------------------------------------------------ gridding (tile gather)
// One CTA owns a 4x4x4 tile of the oversampled grid and up to 16*CG columns.
// Thread (row, g): row = (pz, py) of the tile (16 rows, each 4 x-points),
// g = column group of CG consecutive columns.  The plan holds, per tile, the
// list of samples whose KB support meets it (in sorted-sample order) with the
// tap offsets of the tile origin, so a CTA only stages those samples' weights
// and dcf-weighted values in shared memory, 64 at a time, and every
// (point, column) accumulator sums them in list order: no atomics, bitwise
// reproducible.  The launch runs work items first: a tile's list range
// (lists longer than kSplitEntries are cut into ranges whose partial tiles go
// to a scratch buffer, the first range writing the grid), heaviest first; the
// trailing CTAs write zeros into tiles no sample reaches, kZeroTiles each.
// k_spread_reduce then adds the partial tiles to the grid in range order.
constexpr int kTile = 4;
// List entries staged per sub-chunk (= points of kSlabZ z planes of a tile);
// 64 measured 6 % slower than 32 on the 96-column TVME-256 gridding.
constexpr int kSpreadSub = 32;
constexpr int kSlabZ = kSpreadSub / 16;            // z planes per staged piece of a finished tile
static_assert(kSpreadSub % 16 == 0 && 64 % kSpreadSub == 0, "pieces of whole z planes");
constexpr int kZeroTiles = 4;       // empty tiles per zero-fill CTA (plain stores)
constexpr int kZeroTilesTma = 16;   // empty tiles per zero-fill CTA (TMA stores)
constexpr int kSplitEntries = 256;  // longest list range of one work item

struct SpreadArgs {
    const float4* ks;          // bin base (dcf in .w)
    const TapRec* taps;        // bin base
    const int2* list;          // bin base: (sample, packed tap offsets of the tile origin)
    const int32_t* list_start; // bin base [ntiles + 1]
    const int32_t* tile_order; // bin base [ntiles]: busy tiles, then empty tiles
    const int4* work;          // bin base [n_work]: (tile, first entry, end entry, partial slot or -1)
    int n_busy, n_empty, n_work;
    float2* partials;          // [slot][64 points][ncol] partial tiles of split lists
    int* err;                  // device error word (kDevErr* bits)
    int poll;                  // polls before a bounded mbarrier wait gives up
    const float2* vals;        // (M_b, ncol) bin base
    int ncol, cchunk;          // columns per CTA (blockIdx.y selects the chunk)
    int use_dcf;
    float2* grid;              // (OSZ, OSY, OSX, ncol)
    int os0, os1, os2;
    int nt1, nt2;
};

// Packed tap offset of a tile origin: byte i holds (offset + 128) for axis z, y, x.
__host__ __device__ __forceinline__ int pack_rel(int rz, int ry, int rx) {
    return ((rz + 128) & 0xff) | (((ry + 128) & 0xff) << 8) | (((rx + 128) & 0xff) << 16);
}

__device__ __forceinline__ void tile_geometry(const SpreadArgs& a, int tile, int& t0z, int& t0y, int& t0x,
                                              int& Tz, int& Ty, int& Tx) {
    const int tz = tile / (a.nt1 * a.nt2);
    const int trem = tile - tz * a.nt1 * a.nt2;
    const int ty = trem / a.nt2;
    const int tx = trem - ty * a.nt2;
    t0z = tz * kTile;
    t0y = ty * kTile;
    t0x = tx * kTile;
    Tz = min(kTile, a.os0 - t0z);
    Ty = min(kTile, a.os1 - t0y);
    Tx = min(kTile, a.os2 - t0x);
}

// Tile gather.  TMA = true (even column counts, aligned k-space): each
// entry's values arrive by one bulk copy (cp.async.bulk) on an mbarrier, the
// dcf weight folds into the row weights, and finished tiles (and the zero
// tiles) leave by one 4-D TMA store each, clipped at the grid edge by the TMA
// unit.  TMA = false: values staged by plain loads, coalesced warp stores.
template <int CG, bool TMA>
__global__ void __launch_bounds__(256, (CG >= 6 ? 3 : (CG >= 4 ? 4 : 5))) k_spread(SpreadArgs a,
                                                                 const __grid_constant__ CUtensorMap tgrid) {
    extern __shared__ __align__(128) unsigned char smraw_[];
    __shared__ int l_rel[kSpreadSub];
    __shared__ float s_dcf[kSpreadSub];
    __shared__ float s_wzy[kSpreadSub * 16];
    __shared__ __align__(16) float s_wx[kSpreadSub * 4];
    __shared__ __align__(8) uint64_t bar;
    unsigned char* smraw = reinterpret_cast<unsigned char*>(align128(smraw_));
    float* c_w = reinterpret_cast<float*>(smraw);                        // [kSpreadSub][16]
    float2* dq = reinterpret_cast<float2*>(c_w + 16 * kSpreadSub);       // [kSpreadSub][cchunk]
    const int tid = threadIdx.x;
    const int cst = a.cchunk;                                            // row stride of dq

    // the zero-fill CTAs are spread evenly among the work items (CTA b is zero-fill
    // group floor(b nz / T) when that floor steps at b), so store-only CTAs share
    // the SMs with gathering ones instead of running as a tail
    const int zper = TMA ? kZeroTilesTma : kZeroTiles;
    const long long nzc = (a.n_empty + zper - 1) / zper, T = a.n_work + nzc, bb = blockIdx.x;
    const long long zlo = bb * nzc / T, zhi = (bb + 1) * nzc / T;
    if (zhi > zlo) {
        // ---- zero fill of tiles that no sample reaches (all columns, chunk 0 only)
        if (blockIdx.y != 0) return;
        const int z0 = (int)zlo * zper;
        if constexpr (TMA) {
            float4* z4 = reinterpret_cast<float4*>(dq);          // one zero piece [kSpreadSub][cchunk]
            for (int i = tid; i < (kSpreadSub / 2) * cst; i += 256) z4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                for (int zi = z0; zi < min(z0 + zper, a.n_empty); ++zi) {
                    int t0z, t0y, t0x, Tz, Ty, Tx;
                    tile_geometry(a, a.tile_order[a.n_busy + zi], t0z, t0y, t0x, Tz, Ty, Tx);
                    for (int c0 = 0; c0 < a.ncol; c0 += cst)
                        for (int hz = 0; hz < kTile; hz += kSlabZ) tma_store_4d(&tgrid, dq, c0, t0x, t0y, t0z + hz);
                }
                tma_store_commit_and_drain();
            }
        } else {
            const int warp = tid >> 5, lane = tid & 31;
            for (int r = warp; r < zper * 16; r += 8) {
                const int zi = z0 + (r >> 4);
                if (zi >= a.n_empty) break;
                int t0z, t0y, t0x, Tz, Ty, Tx;
                tile_geometry(a, a.tile_order[a.n_busy + zi], t0z, t0y, t0x, Tz, Ty, Tx);
                const int pz = (r >> 2) & 3, py = r & 3;
                if (pz >= Tz || py >= Ty) continue;
                float2* dst = a.grid + (((int64_t)(t0z + pz) * a.os1 + (t0y + py)) * a.os2 + t0x) * a.ncol;
                const int n2 = Tx * a.ncol;
                if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0 && (n2 & 1) == 0) {
                    float4* d4 = reinterpret_cast<float4*>(dst);
                    for (int i = lane; i < (n2 >> 1); i += 32) d4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                } else {
                    for (int i = lane; i < n2; i += 32) dst[i] = make_float2(0.f, 0.f);
                }
            }
        }
        return;
    }

    const int col0 = blockIdx.y * a.cchunk;
    const int ncc = min(a.cchunk, a.ncol - col0);
    const int4 item = a.work[bb - zlo];
    const int tile = item.x, beg = item.y, end = item.z, slot = item.w;
    int t0z, t0y, t0x, Tz, Ty, Tx;
    tile_geometry(a, tile, t0z, t0y, t0x, Tz, Ty, Tx);
    if (TMA && tid == 0) mbar_init(&bar, 1);

    const int row = tid >> 4;          // tile row (z, y) = (row / 4, row % 4)
    const int g = tid & 15;
    // columns g + 16 j (j < CG): a half-warp (one tile row) reads 16 consecutive
    // values of an entry per load, one 128-byte wavefront (with g CG + j the
    // 8 CG-byte stride put groups g and g + 8 on the same banks)
    float2 acc[4][CG];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int j = 0; j < CG; ++j) acc[x][j] = make_float2(0.f, 0.f);

    unsigned phase = 0;
    for (int base = beg; base < end; base += kSpreadSub, phase ^= 1u) {
        const int ns = min(kSpreadSub, end - base);
        if constexpr (TMA) {
            __syncthreads();                       // dq free; the barrier init is visible
            if (tid < 32) {                        // warp 0: one bulk copy per entry
                if (tid == 0) mbar_expect_tx(&bar, (unsigned)(ns * ncc * sizeof(float2)));
                __syncwarp();
                for (int cand = tid; cand < ns; cand += 32) {
                    const int sm = a.list[base + cand].x;
                    bulk_g2s(dq + cand * cst, a.vals + (int64_t)sm * a.ncol + col0, (unsigned)(ncc * sizeof(float2)),
                             &bar);
                }
            }
        }
        if (tid < 4 * ns) {
            const int cand = tid >> 2, part = tid & 3;
            const int2 e = a.list[base + cand];
            reinterpret_cast<float4*>(c_w)[cand * 4 + part] = a.taps[e.x].w[part];
            if (part == 0) {
                l_rel[cand] = e.y;
                s_dcf[cand] = (TMA && a.use_dcf) ? a.ks[e.x].w : 1.0f;
            }
        }
        if constexpr (!TMA) {
            for (int cand = tid >> 5; cand < ns; cand += 8) {     // one warp per entry, lanes over columns
                const int sm = a.list[base + cand].x;
                const float2* src = a.vals + (int64_t)sm * a.ncol + col0;
                const float dw = a.use_dcf ? a.ks[sm].w : 1.0f;
                for (int col = tid & 31; col < ncc; col += 32) dq[cand * cst + col] = cscale(src[col], dw);
            }
        }
        __syncthreads();
        // per entry: the (z, y) weight of each of the 16 tile rows (times the dcf
        // weight on the TMA path) and the x weight of each of the 4 tile columns
        for (int i = tid; i < ns * 20; i += 256) {
            const int cand = i / 20, k = i - cand * 20;
            const int pk = l_rel[cand];
            const float* w = c_w + 16 * cand;
            if (k < 16) {
                const int az = (pk & 0xff) - 128 + (k >> 2);
                const int ay = ((pk >> 8) & 0xff) - 128 + (k & 3);
                s_wzy[cand * 16 + k] =
                    ((unsigned)az <= 4u && (unsigned)ay <= 4u) ? (w[az] * w[5 + ay]) * s_dcf[cand] : 0.f;
            } else {
                const int ax = ((pk >> 16) & 0xff) - 128 + (k - 16);
                s_wx[cand * 4 + (k - 16)] = (unsigned)ax <= 4u ? w[10 + ax] : 0.f;
            }
        }
        if constexpr (TMA) {
            const bool ok = mbar_wait_or_drain(&bar, phase, a.poll);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) atomicOr(a.err, kDevErrTmaWait);
                return;
            }
        } else {
            __syncthreads();
        }
        for (int cc = 0; cc < ns; ++cc) {
            const float wzy = s_wzy[cc * 16 + row];
            if (wzy == 0.f) continue;
            const float4 wx4 = reinterpret_cast<const float4*>(s_wx)[cc];
            const float wx[4] = {wx4.x, wx4.y, wx4.z, wx4.w};
            float2 v[CG];
#pragma unroll
            for (int j = 0; j < CG; ++j) v[j] = (g + 16 * j < ncc) ? dq[cc * cst + g + 16 * j] : make_float2(0.f, 0.f);
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                if (wx[x] == 0.f) continue;
                const float wt = wzy * wx[x];
#pragma unroll
                for (int j = 0; j < CG; ++j) acc[x][j] = cfma_real(wt, v[j], acc[x][j]);
            }
        }
        if constexpr (!TMA) __syncthreads();
    }
    // ---- store the tile in pieces of kSlabZ z planes: each piece is staged as
    // [kSpreadSub points][cchunk] in the value buffer, then leaves as one TMA box,
    // or by coalesced warp stores (one warp per point); a split list's partial tile
    // goes to its slot instead of the grid
    constexpr int kPieceRows = kSpreadSub / 4;            // tile rows (z, y) per piece
    const int warp = tid >> 5, lane = tid & 31;
    const bool vec = ((ncc | a.ncol | col0 | cst) & 1) == 0;
    for (int piece = 0; piece < 64 / kSpreadSub; ++piece) {
        __syncthreads();                                   // dq free (values, or the previous piece)
        if (row / kPieceRows == piece) {
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int j = 0; j < CG; ++j)
                    if (g + 16 * j < ncc) dq[((row % kPieceRows) * 4 + x) * cst + g + 16 * j] = acc[x][j];
        }
        if (TMA && slot < 0) {
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                tma_store_4d(&tgrid, dq, col0, t0x, t0y, t0z + kSlabZ * piece);
                tma_store_commit_and_drain();
            }
            continue;
        }
        __syncthreads();
        for (int hp = warp; hp < kSpreadSub; hp += 8) {
            const int pt = piece * kSpreadSub + hp;
            const int qz = pt >> 4, qy = (pt >> 2) & 3, qx = pt & 3;
            float2* dst;
            if (slot >= 0) {
                dst = a.partials + ((int64_t)slot * 64 + pt) * a.ncol + col0;
            } else {
                if (qz >= Tz || qy >= Ty || qx >= Tx) continue;
                dst = a.grid + (((int64_t)(t0z + qz) * a.os1 + (t0y + qy)) * a.os2 + (t0x + qx)) * a.ncol + col0;
            }
            const float2* src = dq + hp * cst;
            if (vec) {
                for (int c = lane; c < (ncc >> 1); c += 32)
                    reinterpret_cast<float4*>(dst)[c] = reinterpret_cast<const float4*>(src)[c];
            } else {
                for (int c = lane; c < ncc; c += 32) dst[c] = src[c];
            }
        }
    }
}

// Split lists: grid tile += its partial tiles, in range order (one CTA per tile).
__global__ void __launch_bounds__(256) k_spread_reduce(SpreadArgs a, const int4* __restrict__ splits) {
    const int4 sp = splits[blockIdx.x];
    int t0z, t0y, t0x, Tz, Ty, Tx;
    tile_geometry(a, sp.x, t0z, t0y, t0x, Tz, Ty, Tx);
    const int n = 64 * a.ncol;
    for (int i = threadIdx.x; i < n; i += 256) {
        const int pt = i / a.ncol, col = i - pt * a.ncol;
        const int pz = pt >> 4, py = (pt >> 2) & 3, px = pt & 3;
        if (pz >= Tz || py >= Ty || px >= Tx) continue;
        float2* g = a.grid + (((int64_t)(t0z + pz) * a.os1 + (t0y + py)) * a.os2 + (t0x + px)) * a.ncol + col;
        float2 v = *g;
        for (int s = 0; s < sp.z; ++s) v = cadd(v, a.partials[((int64_t)(sp.y + s) * 64 + pt) * a.ncol + col]);
        *g = v;
    }
}

// ------------------------------------------------------------------ sample order conversion
__global__ void k_sort_ksp(const float2* __restrict__ ext, float2* __restrict__ internal, const int32_t* __restrict__ perm,
                           int64_t M, int ncol) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M * ncol) return;
    const int64_t s = i / ncol;
    const int col = (int)(i - s * ncol);
    internal[i] = ext[(int64_t)col * M + perm[s]];
}

__global__ void k_unsort_ksp(const float2* __restrict__ internal, float2* __restrict__ ext, const int32_t* __restrict__ perm,
                             int64_t M, int ncol) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= M * ncol) return;
    const int64_t s = i / ncol;
    const int col = (int)(i - s * ncol);
    ext[(int64_t)col * M + perm[s]] = internal[i];
}

// (Z, Y, X, C) <- (C, Z, Y, X)
__global__ void k_interleave_maps(const float2* __restrict__ src, float2* __restrict__ dst, int64_t N, int C) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * C) return;
    const int64_t v = i / C;
    const int c = (int)(i - v * C);
    dst[i] = src[(int64_t)c * N + v];
}

// ------------------------------------------------------------------ host helpers
static bool factor_radices(int L, int* radix, int* nstages) {
    int n = L, s = 0;
    for (int r : {7, 5, 3}) {
        while (n % r == 0) {
            if (s >= kMaxStages) return false;
            radix[s++] = r;
            n /= r;
        }
    }
    while (n % 8 == 0) {
        if (s >= kMaxStages) return false;
        radix[s++] = 8;
        n /= 8;
    }
    while (n % 4 == 0) {
        if (s >= kMaxStages) return false;
        radix[s++] = 4;
        n /= 4;
    }
    while (n % 2 == 0) {
        if (s >= kMaxStages) return false;
        radix[s++] = 2;
        n /= 2;
    }
    *nstages = s;
    return n == 1;
}

static size_t fft_smem_bytes(int L, int W) { return (size_t)(2 * L * W + L) * sizeof(float2); }

static tr_status set_smem_limit(const void* fn, size_t bytes) {
    if (bytes > 48 * 1024) TR_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return TR_OK;
}

tr_status ensure_nufft_buffers(tr_plan* p, size_t ncol) {
    if (p->bufA && p->buf_cols >= ncol) return TR_OK;
    if (p->bufA) cudaFree(p->bufA);
    if (p->bufB) cudaFree(p->bufB);
    p->bufA = p->bufB = nullptr;
    const size_t gA = (size_t)p->os[0] * p->os[1] * p->os[2] * ncol;
    const size_t gB = (size_t)p->n[0] * p->os[1] * p->os[2] * ncol;
    TR_CUDA(cudaMalloc(&p->bufA, gA * sizeof(float2)));
    TR_CUDA(cudaMalloc(&p->bufB, gB * sizeof(float2)));
    p->workspace_bytes += (int64_t)((gA + gB) * sizeof(float2));
    p->buf_cols = ncol;
    return TR_OK;
}

// cuTensorMapEncodeTiled from the driver, looked up once (no libcuda link).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    });
    return fn;
}

// 3-D map over complex64 data [d2][d1][d0] (8-byte elements), box [1][b1][b0].
// Every tensor map here promotes L2 fills to 256 bytes: a 128-byte row segment
// of a z-pass box then brings in the segment the next CTA reads (the z passes
// measured 2 % faster than with 128-byte promotion, the other passes unchanged).
static bool encode_map_3d(CUtensorMap* m, const void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0,
                          uint32_t b1) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || ((uintptr_t)base & 15) || (d0 * 8) % 16 || b0 > 256 || b1 > 256 || b0 > d0) return false;
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {d0 * 8, d0 * d1 * 8};
    const cuuint32_t box[3] = {b0, b1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_INT64, 3, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps for k_line_tma, or false when the line's geometry does not split
// into the two-box form (odd lengths, unaligned shared-memory box starts, ...).
static bool line_tma_setup(LineArgs& la, int L, int W, int64_t outer, CUtensorMap* tin, CUtensorMap* tout) {
    if (L % 2 || la.Lout % 2 || la.inner % 2 || la.inner < W || la.inner >= (int64_t)INT32_MAX || outer > 65535 ||
        L / 2 > 256 || la.Lout / 2 > 256 || la.p_in > L / 2)
        return false;
    const int half = la.Lout / 2;
    auto pm = [L](int v) {
        v %= L;
        return v < 0 ? v + L : v;
    };
    const int shift = la.h - la.p_out;
    const int kA = pm(-shift), kB = pm(half - shift);
    if (kA + half > L || kB + half > L) return false;
    if (((int64_t)kA * W * 8) % 128 || ((int64_t)kB * W * 8) % 128 || ((int64_t)(L / 2) * W * 8) % 128) return false;
    if (!encode_map_3d(tin, la.in, (uint64_t)la.inner, (uint64_t)la.Lin, (uint64_t)outer, (uint32_t)W, (uint32_t)(L / 2)))
        return false;
    if (!encode_map_3d(tout, la.out, (uint64_t)la.inner, (uint64_t)la.Lout, (uint64_t)outer, (uint32_t)W, (uint32_t)half))
        return false;
    la.kA = kA;
    la.kB = kB;
    return true;
}

// colmask (z passes of bin grids, ncol k-space columns): skip the lines of
// unoccupied tile columns (inverse: write their zeros), see lines_unoccupied.
static tr_status launch_line(tr_plan* p, int axis, const float2* in, float2* out, int64_t outer, int64_t inner,
                             int Lin, int Lout, int p_in, int p_out, bool inv, cudaStream_t st,
                             const uint8_t* colmask = nullptr, int ncol = 0) {
    const FftAxis& A = p->ax[axis];
    LineArgs la;
    la.colmask = colmask;
    la.skip_zero = inv ? 1 : 0;
    la.mcol = ncol;
    la.mosx = p->os[2];
    la.mnt2 = p->ntile[2];
    la.in = in;
    la.out = out;
    la.inner = inner;
    la.Lin = Lin;
    la.Lout = Lout;
    la.p_in = p_in;
    la.p_out = p_out;
    la.h = A.h;
    la.W = p->line_width;
    la.inv = inv;
    la.tw = A.twiddle;
    la.S = stages_of(A);
    la.err = p->dev_err;
    la.poll = p->poll_limit;
    la.kA = la.kB = 0;
    const void* fn = nullptr;
    CUtensorMap tin, tout;
    bool tma = false;
#define TR_LINE_CASE(LV)                                                                                  \
    case LV:                                                                                              \
        la.W = ct_width(LV);                                                                              \
        tma = p->use_tma && line_tma_setup(la, LV, ct_width(LV), outer, &tin, &tout);                     \
        if (tma)                                                                                          \
            fn = inv ? (const void*)k_line_tma<LV, ct_width(LV), true> : (const void*)k_line_tma<LV, ct_width(LV), false>; \
        else                                                                                              \
            fn = inv ? (const void*)k_line_ct<LV, ct_width(LV), true> : (const void*)k_line_ct<LV, ct_width(LV), false>; \
        break;
    switch (A.L) { TR_CT_LENGTHS(TR_LINE_CASE) default: break; }
#undef TR_LINE_CASE
    unsigned nt = (unsigned)line_threads(A.L, la.W);
    // 320-point lines in two passes (radices 20, 16: measured 15 % faster on the y
    // passes of the 160 x 320 x 320 grid); at 160 the two passes (10, 16: 256 and
    // 160 butterflies) measured 10 % slower than the three (5, 8, 4) and are not used
    if (tma && p->two_pass_320 && A.L == 320) {
        fn = inv ? (const void*)k_line_tma<320, 8, true, 1> : (const void*)k_line_tma<320, 8, false, 1>;
        nt = (unsigned)line_threads_p(A.L, la.W, 1);
    }
    if (!fn) fn = (const void*)k_line;
    la.vec16 = ((inner % 2) == 0 && (la.W % 2) == 0 && ((uintptr_t)in % 16) == 0) ? 1 : 0;
    const size_t smem = tma ? line_tma_smem_bytes(A.L, la.W) : fft_smem_bytes(A.L, la.W);
    dim3 grid((unsigned)((inner + la.W - 1) / la.W), (unsigned)outer);
    TR_TRY(set_smem_limit(fn, smem));
    if (tma) {
        void* args[] = {&la, &tin, &tout};
        TR_CUDA(cudaLaunchKernel(fn, grid, dim3(nt), args, smem, st));
    } else {
        void* args[] = {&la};
        TR_CUDA(cudaLaunchKernel(fn, grid, dim3(256), args, smem, st));
    }
    return TR_OK;
}

static int coils_per_cta(int C) { return C <= 32 ? C : 32; }

// ---- stage launchers (shared by the hot path and the profiler) ----
static tr_status stage_fwd_x(tr_plan* p, const float2* images, int64_t img_stride, int n_img, const float2* maps,
                             int C, cudaStream_t st) {
    const int Z = p->n[0], Y = p->n[1], X = p->n[2], OSX = p->os[2];
    FwdXArgs fa;
    fa.img = images;
    fa.img_stride = img_stride;
    fa.maps = maps;
    fa.C = C;
    fa.n_img = n_img;
    fa.Z = Z;
    fa.Y = Y;
    fa.X = X;
    fa.OSX = OSX;
    fa.h = p->ax[2].h;
    fa.pad = p->ax[2].pad;
    // launch shape: compile-time kernels for the listed lengths
    bool ct = false;
#define TR_IS_CT(LV) case LV: ct = true; break;
    switch (OSX) { TR_CT_LENGTHS(TR_IS_CT) default: break; }
#undef TR_IS_CT
    const int Wct = ct_width(OSX);
    const bool pow2C = (C & (C - 1)) == 0;
    if (ct && (C >= Wct || pow2C)) {
        fa.cc = C >= Wct ? Wct : C;
        fa.rows = Wct / fa.cc;
    } else {
        fa.cc = coils_per_cta(C);
        fa.rows = std::max(1, 16 / fa.cc);
    }
    fa.apz = p->ax[0].apod;
    fa.apy = p->ax[1].apod;
    fa.apx = p->ax[2].apod;
    fa.scale = p->fwd_scale;
    fa.tw = p->ax[2].twiddle;
    fa.S = stages_of(p->ax[2]);
    fa.out = p->bufA;
    fa.ncol = n_img * C;
    fa.err = p->dev_err;
    fa.poll = p->poll_limit;
    // TMA variant: one image row x wt coils per CTA (8, or 4 where 8 does not divide C;
    // the second output box then starts (OSX / 2) 32 bytes into the tile: 128-byte aligned
    // when OSX % 8 == 0)
    int wt = C % kTmaXWidth == 0 ? kTmaXWidth : (C % 4 == 0 ? 4 : 0);
    if (wt == 4 && ((int64_t)(OSX / 2) * wt * 8) % 128) wt = 0;
    if (p->use_tma && ct && maps && wt && X % 16 == 0 && X <= 256 && img_stride % 2 == 0 &&
        (int64_t)X * (wt + 1) <= (int64_t)OSX * wt && OSX / 2 <= 256) {
        CUtensorMap timg, tmap, tout;
        const uint64_t nrows = (uint64_t)Z * Y;
        PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
        bool ok = enc != nullptr;
        if (ok) {
            const cuuint64_t dims[3] = {(cuuint64_t)X, nrows, (cuuint64_t)n_img};
            const cuuint64_t strides[2] = {(cuuint64_t)X * 8, (cuuint64_t)img_stride * 8};
            const cuuint32_t box[3] = {(cuuint32_t)X, 1, 1};
            const cuuint32_t estr[3] = {1, 1, 1};
            ok = enc(&timg, CU_TENSOR_MAP_DATA_TYPE_INT64, 3, const_cast<float2*>(images), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        }
        ok = ok && encode_map_3d(&tmap, maps, (uint64_t)C, (uint64_t)X, nrows, (uint32_t)wt, (uint32_t)X);
        ok = ok && encode_map_3d(&tout, p->bufA, (uint64_t)fa.ncol, (uint64_t)OSX, nrows, (uint32_t)wt,
                                 (uint32_t)(OSX / 2));
        const void* tfn = nullptr;
        unsigned nt = 256;
        if (wt == kTmaXWidth) {
#define TR_FWDX_TMA(LV) case LV: tfn = (const void*)k_fwd_x_tma<LV, kTmaXWidth>; break;
            switch (OSX) { TR_CT_LENGTHS(TR_FWDX_TMA) default: break; }
#undef TR_FWDX_TMA
            if (OSX == 320 && p->two_pass_320) {
                tfn = (const void*)k_fwd_x_wide<320, kTmaXWidth>;
                nt = kWideNT;
            }
        } else {
#define TR_FWDX_TMA4(LV) case LV: tfn = (const void*)k_fwd_x_tma<LV, 4>; break;
            switch (OSX) { TR_CT_LENGTHS(TR_FWDX_TMA4) default: break; }
#undef TR_FWDX_TMA4
        }
        if (ok && tfn) {
            const size_t smem = fft_smem_bytes(OSX, wt) + 128;
            TR_TRY(set_smem_limit(tfn, smem));
            dim3 grid((unsigned)(nrows * n_img), 1u, (unsigned)(C / wt));
            void* args[] = {&fa, &timg, &tmap, &tout};
            TR_CUDA(cudaLaunchKernel(tfn, grid, dim3(nt), args, smem, st));
            return TR_OK;
        }
    }
    const int W = fa.rows * fa.cc;
    const size_t smem = fft_smem_bytes(OSX, W);
    // the n_img CTAs of one row block are adjacent, so the coil-map rows they share come from L2
    dim3 grid((unsigned)(((Z * Y + fa.rows - 1) / fa.rows) * n_img), 1u, (unsigned)((C + fa.cc - 1) / fa.cc));
    const void* fn = nullptr;
    // staged variant when a row's coil-map slice fits the free FFT buffer
    const bool staged = ct && W == Wct && fa.cc >= 4 && (size_t)fa.rows * X * (fa.cc + 1) <= (size_t)OSX * W;
#define TR_FWDX_CASE(LV)                                                                              \
    case LV: {                                                                                        \
        constexpr int WV = ct_width(LV);                                                              \
        if (staged) fn = fa.cc == 16 ? (const void*)k_fwd_x_st<LV, WV, (WV >= 16 ? 16 : WV)>          \
                       : fa.cc == 8 ? (const void*)k_fwd_x_st<LV, WV, 8> : (const void*)k_fwd_x_st<LV, WV, 4>; \
        else if (W == WV) fn = (const void*)k_fwd_x_ct<LV, WV>;                                       \
        else if (W == 12 && WV == 16) fn = (const void*)k_fwd_x_ct<LV, 12>;                          \
        break;                                                                                        \
    }
    switch (OSX) { TR_CT_LENGTHS(TR_FWDX_CASE) default: break; }
#undef TR_FWDX_CASE
    if (!fn) fn = (const void*)k_fwd_x;
    TR_TRY(set_smem_limit(fn, smem));
    void* args[] = {&fa};
    TR_CUDA(cudaLaunchKernel(fn, grid, dim3(256), args, smem, st));
    return TR_OK;
}

// ---- fused y + z passes (k_yz_fwd / k_yz_adj)
// 4-D map over complex64 data with dims (d0 contiguous, then d1, d2, d3 with
// the given byte strides, in any order) and box [b3][b2][b1][b0].
static bool encode_map_4d(CUtensorMap* m, const void* base, const uint64_t dims[4], const uint64_t strides[3],
                          const uint32_t box[4]) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || ((uintptr_t)base & 15) || (box[0] * 8) % 16) return false;
    for (int i = 0; i < 4; ++i)
        if (box[i] < 1 || box[i] > 256 || box[i] > dims[i]) return false;
    for (int i = 0; i < 3; ++i)
        if (strides[i] % 16 || strides[i] >= (1ULL << 40)) return false;
    const cuuint64_t d[4] = {dims[0], dims[1], dims[2], dims[3]};
    const cuuint64_t s[3] = {strides[0], strides[1], strides[2]};
    const cuuint32_t b[4] = {box[0], box[1], box[2], box[3]};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_INT64, 4, const_cast<void*>(base), d, s, b, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The compiled fused shapes: (LY, LZ, cluster size, image rows per CTA): the
// 256 x 256 x 128 and 128 x 128 x 96 workloads' grids.
#define TR_YZ_SHAPES(X) X(320, 160, 16, 8) X(160, 120, 8, 12)

// Fused launch of the forward y + z (adj = false) or adjoint z + y passes on
// plan buffer A in place; *done = false (nothing launched) when the plan, the
// geometry or the device does not allow it, and the caller runs the separate
// passes.
static tr_status stage_yz(tr_plan* p, int ncol, bool adj, cudaStream_t st, bool* done) {
    *done = false;
    const int Z = p->n[0], Y = p->n[1], OSZ = p->os[0], OSY = p->os[1], OSX = p->os[2];
    if (!p->use_tma || !p->fuse_yz || ncol % kYzCW || Z % 2 || Y % 2 || Y / 2 > 256) return TR_OK;
    if (OSY == 320 && !p->two_pass_320) return TR_OK;
    const void* fn = nullptr;
    int CL = 0, ZR = 0;
#define TR_YZ_PICK(LY, LZ, CLV, ZRV)                                                                   \
    if (!fn && OSY == LY && OSZ == LZ && Z == CLV * ZRV) {                                             \
        fn = adj ? (const void*)k_yz_adj<LY, LZ, CLV, ZRV> : (const void*)k_yz_fwd<LY, LZ, CLV, ZRV>;   \
        CL = CLV;                                                                                      \
        ZR = ZRV;                                                                                      \
    }
    TR_YZ_SHAPES(TR_YZ_PICK)
#undef TR_YZ_PICK
    if (!fn) return TR_OK;
    const uint64_t n8 = (uint64_t)ncol * 8;
    // image-side volume (Z, Y, OSX, ncol) viewed as (c, z, y, x); grid (OSZ, OSY, OSX, ncol) as (c, y, z, x)
    const uint64_t img_dims[4] = {(uint64_t)ncol, (uint64_t)Z, (uint64_t)Y, (uint64_t)OSX};
    const uint64_t img_str[3] = {(uint64_t)Y * OSX * n8, (uint64_t)OSX * n8, n8};
    const uint64_t grid_dims[4] = {(uint64_t)ncol, (uint64_t)OSY, (uint64_t)OSZ, (uint64_t)OSX};
    const uint64_t grid_str[3] = {(uint64_t)OSX * n8, (uint64_t)OSY * OSX * n8, n8};
    const uint32_t img_box[4] = {(uint32_t)kYzCW, (uint32_t)ZR, (uint32_t)(adj ? Y / 2 : OSY / 2), 1};
    const uint32_t grid_box[4] = {(uint32_t)kYzCW, 2, (uint32_t)(OSZ / 2), 1};
    CUtensorMap timg, tgrid;
    if (!encode_map_4d(&timg, p->bufA, img_dims, img_str, img_box) ||
        !encode_map_4d(&tgrid, p->bufA, grid_dims, grid_str, grid_box))
        return TR_OK;
    const size_t smem = yz_smem_bytes(OSY, OSZ, ZR);
    TR_TRY(set_smem_limit(fn, smem));
    if (CL > 8) TR_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((int64_t)OSX * (ncol / kYzCW) * CL));
    cfg.blockDim = dim3((unsigned)kYzNT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();                 // the device cannot hold such a cluster: separate passes
        return TR_OK;
    }
    YzArgs ya;
    ya.Z = Z;
    ya.Y = Y;
    ya.pad_z = p->ax[0].pad;
    ya.pad_y = p->ax[1].pad;
    ya.ncol = ncol;
    ya.twz = p->ax[0].twiddle;
    ya.twy = p->ax[1].twiddle;
    ya.err = p->dev_err;
    ya.poll = p->poll_limit;
    void* args[] = {&ya, adj ? (void*)&tgrid : (void*)&timg, adj ? (void*)&timg : (void*)&tgrid};
    TR_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
    *done = true;
    return TR_OK;
}

// y pass: [Z][Y -> OSY][OSX * ncol]
static tr_status stage_fwd_y(tr_plan* p, int ncol, cudaStream_t st) {
    return launch_line(p, 1, p->bufA, p->bufB, p->n[0], (int64_t)p->os[2] * ncol, p->n[1], p->os[1], p->ax[1].pad, 0,
                       false, st);
}

static bool ct_compiled(int L) {
    switch (L) {
#define TR_CT_CASE_TRUE(LV) case LV: return true;
        TR_CT_LENGTHS(TR_CT_CASE_TRUE)
#undef TR_CT_CASE_TRUE
        default: return false;
    }
}

// Unoccupied-column mask of a bin for its z passes and its gridding (null: no
// skipping).  Gridding leaves the tiles of unoccupied columns unwritten only
// when no z-pass CTA mixes lines of occupied and unoccupied columns (a mixed
// CTA transforms all its lines): every CTA's W lines lie in one (y, x) column
// when ncol is a multiple of the z pass's W (16 at the compiled lengths, the
// runtime-radix width elsewhere).
static const uint8_t* bin_colmask(const tr_plan* p, int bin, int ncol) {
    const int zw = ct_compiled(p->os[0]) ? ct_width(p->os[0]) : p->line_width;
    if (!p->skip_empty_cols || !p->colmask || ncol % zw) return nullptr;
    return p->colmask + (int64_t)bin * p->ntile[1] * p->ntile[2];
}

// z pass: [1][Z -> OSZ][OSY * OSX * ncol]; the lines of unoccupied columns are
// not computed (interpolation reads none of them)
static tr_status stage_fwd_z(tr_plan* p, int bin, int ncol, cudaStream_t st) {
    return launch_line(p, 0, p->bufB, p->bufA, 1, (int64_t)p->os[1] * p->os[2] * ncol, p->n[0], p->os[0],
                       p->ax[0].pad, 0, false, st, bin_colmask(p, bin, ncol), ncol);
}

static tr_status stage_interp(tr_plan* p, int bin, int ncol, int mode, float sigma, const float2* y, float2* out,
                              cudaStream_t st) {
    const Bin& b = p->bins[bin];
    if (b.count == 0) return TR_OK;
    int G = 1;
    while (G < ncol && G < 32) G <<= 1;
    const int cpl = (ncol + G - 1) / G;
    const int64_t threads = b.count * G;
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    const TapRec* taps = reinterpret_cast<const TapRec*>(p->taps) + b.offset;
#define TR_INTERP(CPLV)                                                                                      \
    k_interp<CPLV><<<blocks, 256, 0, st>>>(p->bufA, taps, b.count, ncol, G, p->os[0], p->os[1], p->os[2], mode, \
                                           sigma, y, out)
    if (cpl <= 1) TR_INTERP(1);
    else if (cpl <= 2) TR_INTERP(2);
    else if (cpl <= 3) TR_INTERP(3);
    else if (cpl <= 4) TR_INTERP(4);
    else if (cpl <= 8) TR_INTERP(8);
    else return fail(TR_ERR_UNSUPPORTED, "more than 256 k-space columns per bin are not supported");
#undef TR_INTERP
    TR_CHECK_LAUNCH();
    return TR_OK;
}

template <int CG, bool TMA>
static tr_status launch_spread_t(const SpreadArgs& sa, const CUtensorMap& tgrid, unsigned nx, unsigned nchunks,
                                 cudaStream_t st) {
    const size_t smem = (size_t)kSpreadSub * 16 * sizeof(float) + (size_t)kSpreadSub * sa.cchunk * sizeof(float2) + 128;
    const void* fn = (const void*)k_spread<CG, TMA>;
    TR_TRY(set_smem_limit(fn, smem));
    SpreadArgs args_copy = sa;
    CUtensorMap map_copy = tgrid;
    void* args[] = {&args_copy, &map_copy};
    TR_CUDA(cudaLaunchKernel(fn, dim3(nx, nchunks), dim3(256), args, smem, st));
    return TR_OK;
}

// gridding: one CTA per (busy 4x4x4 tile, chunk of <= 128 columns), then the zero-fill CTAs
static tr_status stage_spread(tr_plan* p, int bin, const float2* ksp, int ncol, bool use_dcf, cudaStream_t st) {
    const Bin& b = p->bins[bin];
    SpreadArgs sa;
    sa.ks = p->ks + b.offset;
    sa.taps = reinterpret_cast<const TapRec*>(p->taps) + b.offset;
    sa.list = p->glist + b.list_offset;
    sa.list_start = p->list_start + (int64_t)bin * (p->ntiles + 1);
    sa.tile_order = p->tile_order + (int64_t)bin * p->ntiles;
    sa.work = p->work + b.work_offset;
    sa.n_busy = (int)b.n_busy;
    // zero tiles: only those of occupied columns when the z pass skips the rest
    sa.n_empty = (int)(bin_colmask(p, bin, ncol) ? b.n_zero : p->ntiles - b.n_busy);
    sa.n_work = (int)b.n_work;
    sa.partials = p->bufB;     // free during gridding (the adjoint z pass fills it afterwards)
    sa.vals = ksp;
    sa.ncol = ncol;
    const int nch = (ncol + p->spread_cols - 1) / p->spread_cols;
    sa.cchunk = (ncol + nch - 1) / nch;
    if (nch > 1 && (sa.cchunk & 1)) ++sa.cchunk;     // even chunks keep TMA boxes aligned
    sa.use_dcf = (use_dcf && p->has_dcf) ? 1 : 0;
    sa.grid = p->bufA;
    sa.os0 = p->os[0];
    sa.os1 = p->os[1];
    sa.os2 = p->os[2];
    sa.nt1 = p->ntile[1];
    sa.nt2 = p->ntile[2];
    sa.err = p->dev_err;
    sa.poll = p->poll_limit;
    const int cg = (sa.cchunk + 15) / 16;
    // TMA path: even column counts and chunks, 16-byte aligned k-space rows, an encodable grid map
    CUtensorMap tgrid;
    std::memset(&tgrid, 0, sizeof(tgrid));
    bool tma = p->use_tma && (ncol % 2) == 0 && (sa.cchunk % 2) == 0 && ((uintptr_t)ksp % 16) == 0;
    if (tma) {
        PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
        const cuuint64_t dims[4] = {(cuuint64_t)ncol, (cuuint64_t)p->os[2], (cuuint64_t)p->os[1], (cuuint64_t)p->os[0]};
        const cuuint64_t strides[3] = {(cuuint64_t)ncol * 8, (cuuint64_t)ncol * 8 * p->os[2],
                                       (cuuint64_t)ncol * 8 * p->os[2] * p->os[1]};
        const cuuint32_t box[4] = {(cuuint32_t)sa.cchunk, kTile, kTile, kSlabZ};   // one staged piece
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        tma = enc && enc(&tgrid, CU_TENSOR_MAP_DATA_TYPE_INT64, 4, p->bufA, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    }
    const int zper = tma ? kZeroTilesTma : kZeroTiles;
    const unsigned nx = (unsigned)(sa.n_work + (sa.n_empty + zper - 1) / zper);
#define TR_SPREAD_CG(CGV)                                                    \
    TR_TRY((tma ? launch_spread_t<CGV, true>(sa, tgrid, nx, nch, st)         \
                : launch_spread_t<CGV, false>(sa, tgrid, nx, nch, st)))
    if (cg <= 1) TR_SPREAD_CG(1);
    else if (cg <= 2) TR_SPREAD_CG(2);
    else if (cg <= 3) TR_SPREAD_CG(3);
    else if (cg <= 4) TR_SPREAD_CG(4);
    else if (cg <= 6) TR_SPREAD_CG(6);
    else TR_SPREAD_CG(8);
#undef TR_SPREAD_CG
    if (b.n_split > 0) {
        k_spread_reduce<<<(unsigned)b.n_split, 256, 0, st>>>(sa, p->splits + b.split_offset);
        TR_CHECK_LAUNCH();
    }
    return TR_OK;
}

// z pass (inverse, crop to Z): [1][OSZ -> Z][OSY * OSX * ncol]; the lines of
// unoccupied columns (gridding left them unwritten: they are zero) give zeros
static tr_status stage_adj_z(tr_plan* p, int bin, int ncol, cudaStream_t st) {
    return launch_line(p, 0, p->bufA, p->bufB, 1, (int64_t)p->os[1] * p->os[2] * ncol, p->os[0], p->n[0], 0,
                       p->ax[0].pad, true, st, bin_colmask(p, bin, ncol), ncol);
}

// y pass (inverse, crop to Y): [Z][OSY -> Y][OSX * ncol]
static tr_status stage_adj_y(tr_plan* p, int ncol, cudaStream_t st) {
    return launch_line(p, 1, p->bufB, p->bufA, p->n[0], (int64_t)p->os[2] * ncol, p->os[1], p->n[1], 0,
                       p->ax[1].pad, true, st);
}

// x pass with crop, apodisation and the coil combine
static tr_status stage_adj_x(tr_plan* p, int n_img, const float2* maps, int C, float2* images, int64_t img_stride,
                             cudaStream_t st) {
    const int Z = p->n[0], Y = p->n[1], X = p->n[2], OSX = p->os[2];
    AdjXArgs aa;
    aa.in = p->bufA;
    aa.ncol = n_img * C;
    aa.n_img = n_img;
    aa.maps = maps;
    aa.C = C;
    bool ct = false;
#define TR_IS_CT(LV) case LV: ct = true; break;
    switch (OSX) { TR_CT_LENGTHS(TR_IS_CT) default: break; }
#undef TR_IS_CT
    const int Wct = ct_width(OSX);
    const bool pow2C = (C & (C - 1)) == 0;
    if (ct && (C >= Wct || pow2C)) {
        aa.cc = C >= Wct ? Wct : C;
        aa.rows = Wct / aa.cc;
    } else {
        aa.cc = coils_per_cta(C);
        aa.rows = std::max(1, 16 / aa.cc);
    }
    aa.Z = Z;
    aa.Y = Y;
    aa.X = X;
    aa.OSX = OSX;
    aa.h = p->ax[2].h;
    aa.pad = p->ax[2].pad;
    aa.apz = p->ax[0].apod;
    aa.apy = p->ax[1].apod;
    aa.apx = p->ax[2].apod;
    aa.scale = p->adj_scale;
    aa.tw = p->ax[2].twiddle;
    aa.S = stages_of(p->ax[2]);
    aa.img = images;
    aa.img_stride = img_stride;
    aa.accumulate = 0;
    aa.err = p->dev_err;
    aa.poll = p->poll_limit;
    // TMA variant: one image row per CTA, coil groups of wt (8, or 4 where 8 does not divide C
    // and the second input box, (OSX / 2) 32-byte rows into the tile, is 128-byte aligned)
    int wt = C % kTmaXWidth == 0 ? kTmaXWidth : (C % 4 == 0 ? 4 : 0);
    if (wt == 4 && ((int64_t)(OSX / 2) * wt * 8) % 128) wt = 0;
    if (p->use_tma && ct && maps && wt && OSX / 2 <= 256 && X <= 256 && X + 4 <= OSX) {
        CUtensorMap tin;
        const void* tfn = nullptr;
        unsigned nt = (unsigned)ct_threads(OSX, wt);
        if (wt == kTmaXWidth) {
#define TR_ADJX_TMA(LV) case LV: tfn = (const void*)k_adj_x_tma<LV, kTmaXWidth>; break;
            switch (OSX) { TR_CT_LENGTHS(TR_ADJX_TMA) default: break; }
#undef TR_ADJX_TMA
            if (OSX == 320 && p->two_pass_320 && X % 16 == 0) {  // X <= 256: kWideXBlocks blocks of 16 per warp
                tfn = (const void*)k_adj_x_wide<320, kTmaXWidth>;
                nt = kWideNT;
            }
        } else {
#define TR_ADJX_TMA4(LV) case LV: tfn = (const void*)k_adj_x_tma<LV, 4>; break;
            switch (OSX) { TR_CT_LENGTHS(TR_ADJX_TMA4) default: break; }
#undef TR_ADJX_TMA4
        }
        if (tfn && encode_map_3d(&tin, p->bufA, (uint64_t)aa.ncol, (uint64_t)OSX, (uint64_t)Z * Y, (uint32_t)wt,
                                 (uint32_t)(OSX / 2))) {
            const size_t smem = fft_smem_bytes(OSX, wt) + 128;
            TR_TRY(set_smem_limit(tfn, smem));
            dim3 grid((unsigned)((int64_t)Z * Y * n_img));
            void* args[] = {&aa, &tin};
            TR_CUDA(cudaLaunchKernel(tfn, grid, dim3(nt), args, smem, st));
            return TR_OK;
        }
    }
    const int W = aa.rows * aa.cc;
    const size_t smem = fft_smem_bytes(OSX, W) + (size_t)aa.rows * X * sizeof(float2);
    dim3 grid((unsigned)(((Z * Y + aa.rows - 1) / aa.rows) * n_img));
    const void* fn = nullptr;
    const bool staged = ct && W == Wct;   // cc is a power of two here
#define TR_ADJX_CASE(LV)                                                                              \
    case LV: {                                                                                        \
        constexpr int WV = ct_width(LV);                                                              \
        if (staged) fn = aa.cc == 16 ? (const void*)k_adj_x_st<LV, WV, (WV >= 16 ? 16 : WV)>          \
                       : aa.cc == 8 ? (const void*)k_adj_x_st<LV, WV, 8>                              \
                       : aa.cc == 4 ? (const void*)k_adj_x_st<LV, WV, 4>                              \
                       : aa.cc == 2 ? (const void*)k_adj_x_st<LV, WV, 2> : (const void*)k_adj_x_st<LV, WV, 1>; \
        else if (W == 12 && WV == 16) fn = (const void*)k_adj_x_ct<LV, 12>;                          \
        break;                                                                                        \
    }
    switch (OSX) { TR_CT_LENGTHS(TR_ADJX_CASE) default: break; }
#undef TR_ADJX_CASE
    if (!fn) fn = (const void*)k_adj_x;
    TR_TRY(set_smem_limit(fn, smem));
    void* args[] = {&aa};
    TR_CUDA(cudaLaunchKernel(fn, grid, dim3(256), args, smem, st));
    return TR_OK;
}

tr_status nufft_forward_cols(tr_plan* p, int bin, const float2* images, int64_t img_stride, int n_img,
                             const float2* maps, int C, int mode, float sigma, const float2* y, float2* out,
                             cudaStream_t st) {
    const int ncol = n_img * C;
    TR_TRY(ensure_nufft_buffers(p, (size_t)ncol));
    TR_TRY(stage_fwd_x(p, images, img_stride, n_img, maps, C, st));
    bool fused = false;
    TR_TRY(stage_yz(p, ncol, false, st, &fused));
    if (!fused) {
        TR_TRY(stage_fwd_y(p, ncol, st));
        TR_TRY(stage_fwd_z(p, bin, ncol, st));
    }
    return stage_interp(p, bin, ncol, mode, sigma, y, out, st);
}

// Launch-shape autotuning (TR_PLAN_AUTOTUNE).  The first gridding of a column
// count, outside stream capture, times k_spread for each candidate column chunk
// on the caller's bin (CUDA events, the fastest of three launches after one warm-up) and
// keeps the fastest for that column count.  The choice cannot change results:
// every grid point sums its list in the same order whatever the chunking.
static tr_status tune_spread_cols(tr_plan* p, int bin, const float2* ksp, int ncol, bool use_dcf, cudaStream_t st) {
    auto it = p->spread_cols_tuned.find(ncol);
    if (it != p->spread_cols_tuned.end()) {
        p->spread_cols = it->second;
        return TR_OK;
    }
    p->spread_cols = 128;
    if (!p->autotune || ncol <= 16) return TR_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    TR_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return TR_OK;
    cudaEvent_t e0, e1;
    TR_CUDA(cudaEventCreate(&e0));
    TR_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_cols = 128, last_chunk = -1;
    tr_status rc = TR_OK;
    for (int cols : {32, 48, 64, 96, 128}) {
        const int nch = (ncol + cols - 1) / cols;
        const int chunk = (ncol + nch - 1) / nch;
        if (chunk == last_chunk) continue;       // same launch shape as the previous candidate
        last_chunk = chunk;
        p->spread_cols = cols;
        rc = stage_spread(p, bin, ksp, ncol, use_dcf, st);
        if (rc != TR_OK) break;
        // the best of three launches timed one by one (two back to back flipped
        // between close candidates from run to run)
        float ms = 1e30f;
        for (int r = 0; r < 3 && rc == TR_OK; ++r) {
            cudaEventRecord(e0, st);
            rc = stage_spread(p, bin, ksp, ncol, use_dcf, st);
            cudaEventRecord(e1, st);
            if (rc != TR_OK || cudaEventSynchronize(e1) != cudaSuccess) break;
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            ms = std::min(ms, t);
        }
        if (rc != TR_OK) break;
        if (ms < best) {
            best = ms;
            best_cols = cols;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    TR_TRY(rc);
    p->spread_cols = best_cols;
    p->spread_cols_tuned[ncol] = best_cols;
    return TR_OK;
}

tr_status nufft_adjoint_cols(tr_plan* p, int bin, const float2* ksp, int n_img, const float2* maps, int C,
                             bool use_dcf, float2* images, int64_t img_stride, cudaStream_t st) {
    const int ncol = n_img * C;
    TR_TRY(ensure_nufft_buffers(p, (size_t)ncol));
    TR_TRY(tune_spread_cols(p, bin, ksp, ncol, use_dcf, st));
    TR_TRY(stage_spread(p, bin, ksp, ncol, use_dcf, st));
    bool fused = false;
    TR_TRY(stage_yz(p, ncol, true, st, &fused));
    if (!fused) {
        TR_TRY(stage_adj_z(p, bin, ncol, st));
        TR_TRY(stage_adj_y(p, ncol, st));
    }
    return stage_adj_x(p, n_img, maps, C, images, img_stride, st);
}

// Per-stage CUDA-event timing of the batched NUFFT of one bin (all E echoes x
// C coils), with the algorithmic bytes each stage must move.
tr_status profile_nufft(tr_plan* p, int bin, int reps, double* ms, double* bytes, cudaStream_t st) {
    const int E = p->E, C = p->C, ncol = E * C;
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    const int64_t G = (int64_t)p->os[0] * p->os[1] * p->os[2];
    const int64_t XP = (int64_t)p->n[0] * p->n[1] * p->os[2];      // x-pass rows x OSX
    const int64_t YP = (int64_t)p->n[0] * p->os[1] * p->os[2];      // y-pass output
    const int64_t M = p->bins[bin].count;
    const double c8 = 8.0;
    if (!p->maps) return fail(TR_ERR_INVALID_ARG, "coil maps not set (tr_plan_set_maps)");
    TR_TRY(ensure_nufft_buffers(p, (size_t)ncol));
    float2 *img = nullptr, *ksp = nullptr, *yk = nullptr;
    TR_CUDA(cudaMalloc(&img, (size_t)E * N * sizeof(float2)));
    TR_CUDA(cudaMalloc(&ksp, (size_t)std::max<int64_t>(M, 1) * ncol * sizeof(float2)));
    TR_CUDA(cudaMalloc(&yk, (size_t)std::max<int64_t>(M, 1) * ncol * sizeof(float2)));
    cudaMemsetAsync(img, 0, (size_t)E * N * sizeof(float2), st);
    cudaMemsetAsync(ksp, 0, (size_t)std::max<int64_t>(M, 1) * ncol * sizeof(float2), st);
    cudaMemsetAsync(yk, 0, (size_t)std::max<int64_t>(M, 1) * ncol * sizeof(float2), st);
    TR_TRY(tune_spread_cols(p, bin, ksp, ncol, true, st));
    bytes[0] = c8 * (E * N + C * N + XP * ncol);
    bytes[1] = c8 * ncol * (XP + YP);
    // z passes with the empty-column skip: only the occupied lines are read (and,
    // forward, written); gridding writes the busy and zero-filled tiles only
    const Bin& bb = p->bins[bin];
    const bool skip = bin_colmask(p, bin, ncol) != nullptr;
    const double fo = skip ? (double)bb.n_occ_cols / ((double)p->ntile[1] * p->ntile[2]) : 1.0;
    const double fg = skip ? (double)(bb.n_busy + bb.n_zero) / (double)p->ntiles : 1.0;
    bytes[2] = c8 * ncol * fo * (YP + G);
    bytes[3] = c8 * (G * ncol + 3 * M * ncol) + 16.0 * M;
    bytes[4] = c8 * (M * ncol + fg * G * ncol) + 16.0 * M;
    bytes[5] = c8 * ncol * (fo * G + YP);
    bytes[6] = c8 * ncol * (YP + XP);
    bytes[7] = c8 * (XP * ncol + C * N + E * N);
    bytes[8] = c8 * ncol * (XP + G);      // fused forward y + z
    bytes[9] = c8 * ncol * (G + XP);      // fused adjoint z + y
    ms[8] = ms[9] = 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    tr_status rs = TR_OK;
    for (int s = 0; s < 10 && rs == TR_OK; ++s) {
        bool fused = true;
        auto run = [&]() -> tr_status {
            switch (s) {
                case 0: return stage_fwd_x(p, img, N, E, p->maps, C, st);
                case 1: return stage_fwd_y(p, ncol, st);
                case 2: return stage_fwd_z(p, bin, ncol, st);
                case 3: return stage_interp(p, bin, ncol, kInterpDualProx, 1.f / 6.f, yk, ksp, st);
                case 4: return stage_spread(p, bin, ksp, ncol, true, st);
                case 5: return stage_adj_z(p, bin, ncol, st);
                case 6: return stage_adj_y(p, ncol, st);
                case 7: return stage_adj_x(p, E, p->maps, C, img, N, st);
                case 8: return stage_yz(p, ncol, false, st, &fused);
                default: return stage_yz(p, ncol, true, st, &fused);
            }
        };
        rs = run();  // warm-up
        if (rs == TR_OK && !fused) {     // the plan runs these as the separate passes
            bytes[s] = 0.0;
            continue;
        }
        if (rs != TR_OK) break;
        cudaEventRecord(e0, st);
        for (int r = 0; r < reps && rs == TR_OK; ++r) rs = run();
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            rs = fail(TR_ERR_CUDA, "profiling failed");
            break;
        }
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms[s] = t / std::max(reps, 1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(img);
    cudaFree(ksp);
    cudaFree(yk);
    return rs;
}

static double apod_value(int i, int n, int L, int width, double beta) {
    const double t = M_PI * width * (double)(i - n / 2) / (double)L;
    const double r = std::sqrt(beta * beta - t * t);
    return r / std::sinh(r);
}

static void plan_free(tr_plan* p) {
    if (!p) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(p->device);
    pdhg_destroy(p);
    wavelet_destroy(p);
    for (auto& a : p->ax) {
        cudaFree(a.twiddle);
        cudaFree(a.apod);
    }
    cudaFree(p->ks);
    cudaFree(p->taps);
    cudaFree(p->perm);
    cudaFree(p->glist);
    cudaFree(p->work);
    cudaFree(p->splits);
    cudaFree(p->list_start);
    cudaFree(p->tile_order);
    cudaFree(p->colmask);
    cudaFree(p->maps);
    cudaFree(p->bufA);
    cudaFree(p->bufB);
    cudaFree(p->one_in);
    cudaFree(p->one_out);
    cudaFree(p->partials);
    cudaFree(p->tol_dev);
    cudaFree(p->dev_err);
    if (p->err_host) cudaFreeHost(p->err_host);
    if (p->tol_host) cudaFreeHost(p->tol_host);
    cudaSetDevice(cur);
    delete p;
}

// Tiles of one axis met by the KB support of coordinate k: the first tap
// ceil(k - 2) (in double, as the device's axis_taps), four taps, and a fifth
// where the device gives it a nonzero weight (|(b0 + 4 - k) / 2| <= 1 in float);
// tiles in order of first appearance with the tap offset of each tile origin.
static int axis_tiles(float k, int os, int* tile, int* rel) {
    const int b0 = (int)std::ceil((double)k - 2.0);
    volatile float d4 = ((float)(b0 + 4) - k) * 0.5f;
    const int nt = std::fabs((float)d4) <= 1.0f ? 5 : 4;
    int n = 0;
    for (int t = 0; t < nt; ++t) {
        int pos = (b0 + t) % os;
        if (pos < 0) pos += os;
        const int tt = pos / kTile;
        bool seen = false;
        for (int i = 0; i < n; ++i) seen |= tile[i] == tt;
        if (seen) continue;
        int r = (tt * kTile - b0) % os;     // tap index of the tile origin, in (-os + 4, 4]
        if (r < 0) r += os;
        if (r > 4) r -= os;
        tile[n] = tt;
        rel[n] = r;
        ++n;
    }
    return n;
}

// Gather lists of one bin (ks: its tile-sorted scaled coordinates): for every
// grid tile the samples whose support meets it, in sorted-sample order, as
// (sample, packed tap offsets); list_start [ntiles + 1] relative to the bin's
// first entry; order: busy tiles by entry count (heaviest first, stable),
// then the empty tiles of occupied (y, x) tile columns, then the rest;
// colmask [ntile[1] * ntile[2]]: 1 for the occupied columns.
static tr_status build_gather_lists(tr_plan* p, int bin, const float4* ks, int64_t M, std::vector<int2>& glist,
                                    int32_t* list_start, int32_t* order, uint8_t* colmask, std::vector<int4>& work,
                                    std::vector<int4>& splits) {
    const int64_t nt = p->ntiles;
    std::vector<int64_t> cnt((size_t)nt + 1, 0);
    auto visit = [&](auto&& emit) {
        for (int64_t m = 0; m < M; ++m) {
            int tz[5], ty[5], tx[5], rz[5], ry[5], rx[5];
            const int nz = axis_tiles(ks[m].x, p->os[0], tz, rz);
            const int ny = axis_tiles(ks[m].y, p->os[1], ty, ry);
            const int nx = axis_tiles(ks[m].z, p->os[2], tx, rx);
            for (int i = 0; i < nz; ++i)
                for (int j = 0; j < ny; ++j)
                    for (int l = 0; l < nx; ++l)
                        emit(((int64_t)tz[i] * p->ntile[1] + ty[j]) * p->ntile[2] + tx[l], (int32_t)m,
                             pack_rel(rz[i], ry[j], rx[l]));
        }
    };
    visit([&](int64_t t, int32_t, int) { cnt[(size_t)t + 1]++; });
    for (int64_t t = 0; t < nt; ++t) cnt[(size_t)t + 1] += cnt[(size_t)t];
    const int64_t total = cnt[(size_t)nt];
    if (total > (int64_t)INT32_MAX)
        return fail(TR_ERR_UNSUPPORTED, "gridding lists of one bin exceed 2^31 entries; split the bin");
    Bin& B = p->bins[bin];
    B.list_offset = (int64_t)glist.size();
    B.list_count = total;
    glist.resize(glist.size() + (size_t)total);
    int2* dst = glist.data() + B.list_offset;
    std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1);
    visit([&](int64_t t, int32_t m, int packed) { dst[cur[(size_t)t]++] = make_int2(m, packed); });
    std::vector<std::pair<int64_t, int32_t>> busy;
    std::vector<int32_t> empty, unoccupied;
    const int64_t ncolumns = (int64_t)p->ntile[1] * p->ntile[2];
    std::fill(colmask, colmask + ncolumns, (uint8_t)0);
    for (int64_t t = 0; t < nt; ++t)
        if (cnt[(size_t)t + 1] > cnt[(size_t)t]) colmask[t % ncolumns] = 1;   // t = tz * ncolumns + column
    B.n_occ_cols = std::count(colmask, colmask + ncolumns, (uint8_t)1);
    for (int64_t t = 0; t < nt; ++t) {
        list_start[t] = (int32_t)cnt[(size_t)t];
        const int64_t c = cnt[(size_t)t + 1] - cnt[(size_t)t];
        if (c > 0) busy.push_back({-c, (int32_t)t});
        else if (colmask[t % ncolumns]) empty.push_back((int32_t)t);
        else unoccupied.push_back((int32_t)t);
    }
    list_start[nt] = (int32_t)total;
    std::stable_sort(busy.begin(), busy.end(),
                     [](const std::pair<int64_t, int32_t>& x, const std::pair<int64_t, int32_t>& y) {
                         return x.first < y.first;
                     });
    B.n_busy = (int64_t)busy.size();
    B.n_zero = (int64_t)empty.size();
    for (size_t i = 0; i < busy.size(); ++i) order[i] = busy[i].second;
    for (size_t i = 0; i < empty.size(); ++i) order[busy.size() + i] = empty[i];
    for (size_t i = 0; i < unoccupied.size(); ++i) order[busy.size() + empty.size() + i] = unoccupied[i];
    // work items: lists longer than `split` entries become ranges of `split`;
    // their partial tiles (64 points x ncol) live in the y-pass buffer, which
    // holds n[0] * os[1] * os[2] points per column, so the split is widened
    // until the partials fit
    const int64_t max_slots = (int64_t)p->n[0] * p->os[1] * p->os[2] / 64;
    int64_t split = kSplitEntries;
    auto extra_slots = [&](int64_t sp) {
        int64_t e = 0;
        for (const auto& w : busy) e += (-w.first + sp - 1) / sp - 1;
        return e;
    };
    while (extra_slots(split) > max_slots) split *= 2;
    B.work_offset = (int64_t)work.size();
    B.split_offset = (int64_t)splits.size();
    int32_t slot = 0;
    for (const auto& w : busy) {
        const int64_t c = -w.first;
        const int32_t t = w.second;
        const int32_t beg = list_start[t];
        const int64_t ns = (c + split - 1) / split;
        if (ns > 1) splits.push_back(make_int4(t, slot, (int)(ns - 1), 0));
        for (int64_t r = 0; r < ns; ++r) {
            const int32_t b0 = beg + (int32_t)(r * split);
            const int32_t b1 = beg + (int32_t)std::min<int64_t>(c, (r + 1) * split);
            work.push_back(make_int4(t, b0, b1, r == 0 ? -1 : slot++));
        }
    }
    B.n_work = (int64_t)work.size() - B.work_offset;
    B.n_split = (int64_t)splits.size() - B.split_offset;
    return TR_OK;
}

static tr_status plan_create_impl(const tr_plan_desc* d, tr_plan** out) {
    if (!d || !out) return fail(TR_ERR_INVALID_ARG, "tr_plan_create: null argument");
    *out = nullptr;
    for (int i = 0; i < 3; ++i)
        if (d->img_shape[i] < 10)
            return fail(TR_ERR_INVALID_ARG, "img_shape must be three values >= 10 (z, y, x)");
    if (d->n_bins < 1 || !d->bin_counts) return fail(TR_ERR_INVALID_ARG, "at least one trajectory bin is required");
    if (d->n_coils < 1 || d->n_echoes < 1) return fail(TR_ERR_INVALID_ARG, "n_coils and n_echoes must be >= 1");
    if (std::fabs(d->oversamp - 1.25f) > 1e-6f || d->width != 4)
        return fail(TR_ERR_UNSUPPORTED, "only oversamp = 1.25 and width = 4 (the reference's SigPy defaults) are supported");
    int ndev = 0;
    TR_CUDA(cudaGetDeviceCount(&ndev));
    if (d->device < 0 || d->device >= ndev) return fail(TR_ERR_INVALID_ARG, "invalid CUDA device ordinal");
    DeviceGuard guard(d->device);

    tr_plan* p = new tr_plan();
    p->device = d->device;
    p->C = d->n_coils;
    p->E = d->n_echoes;
    p->B = d->n_bins;
    p->width = d->width;
    const double beta = M_PI * std::sqrt(std::pow(d->width / (double)d->oversamp * (d->oversamp - 0.5), 2.0) - 0.8);
    p->beta = (float)beta;
    double N = 1.0;
    for (int i = 0; i < 3; ++i) {
        p->n[i] = d->img_shape[i];
        p->os[i] = (int)std::ceil((double)d->oversamp * d->img_shape[i]);
        N *= p->n[i];
    }
    p->fwd_scale = (float)(1.0 / (std::sqrt(N) * std::pow((double)d->width, 3)));
    p->adj_scale = p->fwd_scale;
    // frees the half-built plan on every early return (TR_CUDA / TR_TRY included)
    struct PlanOwner {
        tr_plan* p;
        ~PlanOwner() {
            if (p) plan_free(p);
        }
    } owner{p};
    auto bad = [&](tr_status code, const std::string& m) { return fail(code, m); };
    for (int i = 0; i < 3; ++i) {
        FftAxis& A = p->ax[i];
        A.n = p->n[i];
        A.L = p->os[i];
        A.h = A.L / 2;
        A.pad = A.L / 2 - A.n / 2;
        if (A.L > kMaxFftLen || !factor_radices(A.L, A.radix, &A.nstages))
            return bad(TR_ERR_UNSUPPORTED, "oversampled length " + std::to_string(A.L) +
                                           " must factor into 2, 3, 5, 7 and be <= 1024");
        std::vector<float2> tw(A.L);
        for (int k = 0; k < A.L; ++k) {
            const double ang = -2.0 * M_PI * (double)k / (double)A.L;
            tw[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
        }
        std::vector<float> ap(A.n);
        for (int k = 0; k < A.n; ++k) ap[k] = (float)apod_value(k, A.n, A.L, d->width, beta);
        if (cudaMalloc(&A.twiddle, A.L * sizeof(float2)) != cudaSuccess ||
            cudaMalloc(&A.apod, A.n * sizeof(float)) != cudaSuccess)
            return bad(TR_ERR_OOM, "allocation of FFT tables failed");
        cudaMemcpy(A.twiddle, tw.data(), A.L * sizeof(float2), cudaMemcpyHostToDevice);
        cudaMemcpy(A.apod, ap.data(), A.n * sizeof(float), cudaMemcpyHostToDevice);
        p->ntile[i] = (A.L + kTile - 1) / kTile;
    }
    p->ntiles = (int64_t)p->ntile[0] * p->ntile[1] * p->ntile[2];

    // bins
    p->bins.resize(d->n_bins);
    int64_t off = 0;
    for (int b = 0; b < d->n_bins; ++b) {
        if (d->bin_counts[b] < 0 || d->bin_counts[b] > (int64_t)INT32_MAX)
            return bad(TR_ERR_INVALID_ARG, "bin sample counts must be in [0, 2^31)");
        p->bins[b].offset = off;
        p->bins[b].count = d->bin_counts[b];
        off += d->bin_counts[b];
    }
    p->total = off;
    if (off > 0 && !d->coords) return bad(TR_ERR_INVALID_ARG, "coords is null");
    p->has_dcf = d->dcf != nullptr;

    // scale coordinates exactly as the reference (float32 multiply, then add)
    std::vector<float4> ks_sorted((size_t)std::max<int64_t>(off, 1));
    std::vector<int32_t> perm((size_t)std::max<int64_t>(off, 1));
    std::vector<int32_t> lstart((size_t)(p->ntiles + 1) * d->n_bins);
    std::vector<int32_t> torder((size_t)p->ntiles * d->n_bins);
    const size_t ncolumns = (size_t)p->ntile[1] * p->ntile[2];
    std::vector<uint8_t> cmask(ncolumns * d->n_bins);
    std::vector<int2> glist;
    std::vector<int4> gwork, gsplits;
    float scale[3], shift[3];
    for (int i = 0; i < 3; ++i) {
        scale[i] = (float)((double)p->os[i] / (double)p->n[i]);
        shift[i] = (float)(p->os[i] / 2);
    }
    // per bin (in parallel over host threads): scaled coordinates, stable counting
    // sort by tile, gather lists; bins write disjoint ranges, lists are joined in bin order
    struct BinOut {
        tr_status rc = TR_OK;
        std::string msg;
        std::vector<int2> glist;
        std::vector<int4> work, splits;
    };
    std::vector<BinOut> outs((size_t)d->n_bins);
    auto do_bin = [&](int b) {
        BinOut& out = outs[(size_t)b];
        const int64_t M = p->bins[b].count, o = p->bins[b].offset;
        std::vector<int32_t> key((size_t)M, 0);
        std::vector<float4> kscaled((size_t)M, make_float4(0, 0, 0, 0));
        for (int64_t m = 0; m < M; ++m) {
            float kc[3];
            for (int i = 0; i < 3; ++i) {
                volatile float t = d->coords[(o + m) * 3 + i] * scale[i];
                kc[i] = t + shift[i];
                if (!std::isfinite(kc[i])) {
                    out.rc = TR_ERR_INVALID_ARG;
                    out.msg = "coordinates must be finite";
                    return;
                }
            }
            const float w = d->dcf ? d->dcf[o + m] : 1.0f;
            kscaled[(size_t)m] = make_float4(kc[0], kc[1], kc[2], w);
            int tcoord[3];
            for (int i = 0; i < 3; ++i) {
                long long f = (long long)std::floor((double)kc[i]);
                long long r = f % p->os[i];
                if (r < 0) r += p->os[i];
                tcoord[i] = (int)(r / kTile);
            }
            key[(size_t)m] = (tcoord[0] * p->ntile[1] + tcoord[1]) * p->ntile[2] + tcoord[2];
        }
        // stable counting sort by tile
        std::vector<int32_t> ts((size_t)p->ntiles + 1, 0);
        for (int64_t m = 0; m < M; ++m) ts[(size_t)key[(size_t)m] + 1]++;
        for (int64_t t = 0; t < p->ntiles; ++t) ts[(size_t)t + 1] += ts[(size_t)t];
        std::vector<int32_t> fillp(ts.begin(), ts.end() - 1);
        for (int64_t m = 0; m < M; ++m) {
            const int32_t pos = fillp[(size_t)key[(size_t)m]]++;
            perm[(size_t)(o + pos)] = (int32_t)m;
            ks_sorted[(size_t)(o + pos)] = kscaled[(size_t)m];
        }
        // gather lists: every (tile, sample) pair where the sample's KB support meets the tile
        out.rc = build_gather_lists(p, b, M ? &ks_sorted[(size_t)o] : nullptr, M, out.glist,
                                    &lstart[(size_t)b * (p->ntiles + 1)], &torder[(size_t)b * p->ntiles],
                                    &cmask[(size_t)b * ncolumns], out.work, out.splits);
        if (out.rc != TR_OK) out.msg = g_last_error;     // this worker thread's message
    };
    {
        std::atomic<int> next_bin{0};
        auto worker = [&]() {
            for (int b; (b = next_bin++) < d->n_bins;) {
                try {
                    do_bin(b);
                } catch (const std::exception& e) {
                    outs[(size_t)b].rc = TR_ERR_OOM;
                    outs[(size_t)b].msg = std::string("plan creation: ") + e.what();
                }
            }
        };
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const int nthr = (int)std::min<unsigned>(hw, (unsigned)d->n_bins);
        std::vector<std::thread> pool;
        for (int i = 1; i < nthr; ++i) pool.emplace_back(worker);
        worker();
        for (auto& t : pool) t.join();
    }
    for (int b = 0; b < d->n_bins; ++b) {
        BinOut& out = outs[(size_t)b];
        if (out.rc != TR_OK) return bad(out.rc, out.msg);
        Bin& B = p->bins[b];
        B.list_offset = (int64_t)glist.size();
        B.work_offset = (int64_t)gwork.size();
        B.split_offset = (int64_t)gsplits.size();
        glist.insert(glist.end(), out.glist.begin(), out.glist.end());
        gwork.insert(gwork.end(), out.work.begin(), out.work.end());
        gsplits.insert(gsplits.end(), out.splits.begin(), out.splits.end());
        std::vector<int2>().swap(out.glist);
    }
    const size_t nks = (size_t)std::max<int64_t>(off, 1);
    if (cudaMalloc(&p->ks, nks * sizeof(float4)) != cudaSuccess ||
        cudaMalloc(&p->taps, nks * sizeof(TapRec)) != cudaSuccess ||
        cudaMalloc(&p->perm, nks * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&p->glist, std::max<size_t>(glist.size(), 1) * sizeof(int2)) != cudaSuccess ||
        cudaMalloc(&p->list_start, lstart.size() * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&p->work, std::max<size_t>(gwork.size(), 1) * sizeof(int4)) != cudaSuccess ||
        cudaMalloc(&p->splits, std::max<size_t>(gsplits.size(), 1) * sizeof(int4)) != cudaSuccess ||
        cudaMalloc(&p->tile_order, torder.size() * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&p->colmask, cmask.size()) != cudaSuccess)
        return bad(TR_ERR_OOM, "allocation of the sorted trajectory failed");
    TR_CUDA(cudaMemcpy(p->ks, ks_sorted.data(), nks * sizeof(float4), cudaMemcpyHostToDevice));
    TR_CUDA(cudaMemcpy(p->perm, perm.data(), nks * sizeof(int32_t), cudaMemcpyHostToDevice));
    k_prep_taps<<<(unsigned)((nks + 255) / 256), 256>>>(p->ks, (int64_t)nks, p->beta, (TapRec*)p->taps);
    TR_CHECK_LAUNCH();
    TR_CUDA(cudaDeviceSynchronize());
    if (!glist.empty())
        TR_CUDA(cudaMemcpy(p->glist, glist.data(), glist.size() * sizeof(int2), cudaMemcpyHostToDevice));
    TR_CUDA(cudaMemcpy(p->list_start, lstart.data(), lstart.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    if (!gwork.empty())
        TR_CUDA(cudaMemcpy(p->work, gwork.data(), gwork.size() * sizeof(int4), cudaMemcpyHostToDevice));
    if (!gsplits.empty())
        TR_CUDA(cudaMemcpy(p->splits, gsplits.data(), gsplits.size() * sizeof(int4), cudaMemcpyHostToDevice));
    TR_CUDA(cudaMemcpy(p->tile_order, torder.data(), torder.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    TR_CUDA(cudaMemcpy(p->colmask, cmask.data(), cmask.size(), cudaMemcpyHostToDevice));
    if (cudaMalloc(&p->tol_dev, 4 * sizeof(double)) != cudaSuccess ||
        cudaMallocHost(&p->tol_host, 4 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&p->dev_err, sizeof(int)) != cudaSuccess || cudaMallocHost(&p->err_host, sizeof(int)) != cudaSuccess)
        return bad(TR_ERR_OOM, "allocation of reduction scalars failed");
    TR_CUDA(cudaMemset(p->dev_err, 0, sizeof(int)));
    *p->err_host = 0;
    p->use_tma = (d->flags & TR_PLAN_NO_TMA) == 0;
    p->fuse_yz = (d->flags & TR_PLAN_YZ_FUSION) != 0;
    p->two_pass_320 = (d->flags & TR_PLAN_THREE_PASS_320) == 0;
    // the fused y + z kernels transform every line: gridding then zero-fills every empty tile
    p->skip_empty_cols = (d->flags & TR_PLAN_NO_COLUMN_SKIP) == 0 && !p->fuse_yz;
    p->autotune = (d->flags & TR_PLAN_AUTOTUNE) != 0;
    p->workspace_bytes = (int64_t)(nks * (sizeof(float4) + sizeof(TapRec) + sizeof(int32_t)) +
                                   glist.size() * sizeof(int2) + (gwork.size() + gsplits.size()) * sizeof(int4) +
                                   (lstart.size() + torder.size()) * sizeof(int32_t) + cmask.size());
    TR_TRY(wavelet_prepare(p));
    owner.p = nullptr;
    *out = p;
    return TR_OK;
}

}  // namespace tr

using namespace tr;

extern "C" {

const char* tr_last_error_string(void) { return g_last_error.c_str(); }

tr_status tr_plan_create(const tr_plan_desc* desc, tr_plan** out) {
    try {
        return plan_create_impl(desc, out);
    } catch (const std::exception& e) {
        return fail(TR_ERR_OOM, std::string("tr_plan_create: ") + e.what());
    }
}

tr_status tr_plan_destroy(tr_plan* plan) {
    if (!plan) return TR_OK;
    plan_free(plan);
    return TR_OK;
}

tr_status tr_plan_info(const tr_plan* p, tr_plan_info_t* info) {
    if (!p || !info) return fail(TR_ERR_INVALID_ARG, "tr_plan_info: null argument");
    for (int i = 0; i < 3; ++i) info->os_shape[i] = p->os[i];
    info->total_samples = p->total;
    info->workspace_bytes = p->workspace_bytes;
    info->fft_line_width = p->line_width;
    info->spread_columns = p->spread_cols;
    info->wavelet_levels = 0;
    info->wavelet_coeffs = 0;
    wavelet_info(p, &info->wavelet_levels, &info->wavelet_coeffs);
    return TR_OK;
}

tr_status tr_plan_set_wait_limit(tr_plan* p, int32_t polls) {
    if (!p) return fail(TR_ERR_INVALID_ARG, "tr_plan_set_wait_limit: null plan");
    if (polls < 0) return fail(TR_ERR_INVALID_ARG, "tr_plan_set_wait_limit: polls must be >= 0");
    p->poll_limit = polls;
    pdhg_destroy(p);   // a captured iteration holds the old limit in its kernel parameters
    return TR_OK;
}

tr_status tr_plan_bin_offset(const tr_plan* p, int32_t bin, int64_t* offset, int64_t* count) {
    if (!p) return fail(TR_ERR_INVALID_ARG, "null plan");
    if (bin < 0 || bin >= p->B)
        return fail(TR_ERR_INVALID_ARG, "bin_index " + std::to_string(bin) + " is outside [0, " +
                                            std::to_string(p->B) + ").");
    if (offset) *offset = p->bins[bin].offset;
    if (count) *count = p->bins[bin].count;
    return TR_OK;
}

tr_status tr_plan_set_maps(tr_plan* p, const void* mps, void* stream) {
    if (!p || !mps) return fail(TR_ERR_INVALID_ARG, "tr_plan_set_maps: null argument");
    DeviceGuard g(p->device);
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    if (!p->maps) {
        TR_CUDA(cudaMalloc(&p->maps, (size_t)N * p->C * sizeof(float2)));
        p->workspace_bytes += N * p->C * (int64_t)sizeof(float2);
    }
    const int64_t tot = N * p->C;
    k_interleave_maps<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>((const float2*)mps, p->maps,
                                                                                        N, p->C);
    TR_CHECK_LAUNCH();
    return TR_OK;
}

tr_status tr_plan_sort_kspace(tr_plan* p, int32_t bin, const void* ext, void* internal, int32_t ncol,
                              void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!ext || !internal || ncol < 1) return fail(TR_ERR_INVALID_ARG, "tr_plan_sort_kspace: bad argument");
    DeviceGuard g(p->device);
    const Bin& b = p->bins[bin];
    const int64_t n = b.count * ncol;
    if (n == 0) return TR_OK;
    k_sort_ksp<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const float2*)ext, (float2*)internal, p->perm + b.offset, b.count, ncol);
    TR_CHECK_LAUNCH();
    return TR_OK;
}

tr_status tr_plan_unsort_kspace(tr_plan* p, int32_t bin, const void* internal, void* ext, int32_t ncol,
                                void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!ext || !internal || ncol < 1) return fail(TR_ERR_INVALID_ARG, "tr_plan_unsort_kspace: bad argument");
    DeviceGuard g(p->device);
    const Bin& b = p->bins[bin];
    const int64_t n = b.count * ncol;
    if (n == 0) return TR_OK;
    k_unsort_ksp<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        (const float2*)internal, (float2*)ext, p->perm + b.offset, b.count, ncol);
    TR_CHECK_LAUNCH();
    return TR_OK;
}

static tr_status ensure_one(tr_plan* p) {
    size_t need = (size_t)std::max<int64_t>(1, 0);
    for (auto& b : p->bins) need = std::max(need, (size_t)b.count);
    if (p->one_in && p->one_elems >= need) return TR_OK;
    cudaFree(p->one_in);
    cudaFree(p->one_out);
    p->one_in = p->one_out = nullptr;
    TR_CUDA(cudaMalloc(&p->one_in, need * sizeof(float2)));
    TR_CUDA(cudaMalloc(&p->one_out, need * sizeof(float2)));
    p->one_elems = need;
    return TR_OK;
}

tr_status tr_nufft_forward(tr_plan* p, int32_t bin, const void* image, void* ksp, void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!image || !ksp) return fail(TR_ERR_INVALID_ARG, "tr_nufft_forward: null pointer");
    DeviceGuard g(p->device);
    TR_TRY(ensure_one(p));
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    TR_TRY(nufft_forward_cols(p, bin, (const float2*)image, N, 1, nullptr, 1, kInterpStore, 0.f, nullptr,
                              p->one_out, st));
    return tr_plan_unsort_kspace(p, bin, p->one_out, ksp, 1, stream);
}

tr_status tr_nufft_adjoint(tr_plan* p, int32_t bin, const void* ksp, void* image, void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!image || !ksp) return fail(TR_ERR_INVALID_ARG, "tr_nufft_adjoint: null pointer");
    DeviceGuard g(p->device);
    TR_TRY(ensure_one(p));
    cudaStream_t st = (cudaStream_t)stream;
    TR_TRY(tr_plan_sort_kspace(p, bin, ksp, p->one_in, 1, stream));
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    return nufft_adjoint_cols(p, bin, p->one_in, 1, nullptr, 1, false, (float2*)image, N, st);
}

tr_status tr_nufft_forward_bin(tr_plan* p, int32_t bin, const void* images, void* ksp_internal, void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!images || !ksp_internal) return fail(TR_ERR_INVALID_ARG, "tr_nufft_forward_bin: null pointer");
    if (!p->maps) return fail(TR_ERR_INVALID_ARG, "coil maps not set (tr_plan_set_maps)");
    DeviceGuard g(p->device);
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    return nufft_forward_cols(p, bin, (const float2*)images, N, p->E, p->maps, p->C, kInterpStore, 0.f, nullptr,
                              (float2*)ksp_internal, (cudaStream_t)stream);
}

tr_status tr_profile_nufft(tr_plan* p, int32_t bin, int32_t reps, double* ms, double* bytes, void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!ms || !bytes || reps < 1) return fail(TR_ERR_INVALID_ARG, "tr_profile_nufft: bad argument");
    DeviceGuard g(p->device);
    return profile_nufft(p, bin, reps, ms, bytes, (cudaStream_t)stream);
}

tr_status tr_nufft_adjoint_bin(tr_plan* p, int32_t bin, const void* ksp_internal, int32_t use_dcf, void* images,
                               void* stream) {
    TR_TRY(tr_plan_bin_offset(p, bin, nullptr, nullptr));
    if (!images || !ksp_internal) return fail(TR_ERR_INVALID_ARG, "tr_nufft_adjoint_bin: null pointer");
    if (!p->maps) return fail(TR_ERR_INVALID_ARG, "coil maps not set (tr_plan_set_maps)");
    DeviceGuard g(p->device);
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    return nufft_adjoint_cols(p, bin, (const float2*)ksp_internal, p->E, p->maps, p->C, use_dcf != 0,
                              (float2*)images, N, (cudaStream_t)stream);
}

}  // extern "C"
