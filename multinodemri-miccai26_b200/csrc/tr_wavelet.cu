// TVMW spatial wavelet W2 on sm_100a: db6, PyWavelets "zero" mode, level =
// PyWavelets' maximum, over (Z, Y, X) of every (bin, echo) image.
//
// Reference: src/toporecon/algorithms/tvmw.py:196-206 (ptwt wavedec3 /
// waverec3, axes (-3, -2, -1)), the dual step at :447-452 (p += sigma W2 u,
// then _tree_project_linf_complex2ch_ at :162-193 on every sub-band), and the
// primal use of waverec3 as the adjoint substitute at :647-649.
//
// Analysis along one axis:   c[o] = sum_j f[j] x[2o + 1 - j], x = 0 outside,
//                            output length (n + F - 1) / 2.
// Synthesis along one axis:  y[o] = sum_j g_lo[2j + o%2] a[i - j] + g_hi[2j + o%2] d[i - j],
//                            i = o/2 + F/2 - 1, computed only for the lengths
//                            the next finer level needs (PyWavelets' crop).
// Coefficients of one image: [cA_L | 7 detail bands of level L | ... | level 1],
// detail bands ordered aad, ada, add, daa, dad, dda, ddd (z, y, x letters).

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <vector>

#include "tr_internal.cuh"

namespace tr {

constexpr int kF = 12;          // db6 filter length
constexpr int kMaxLevels = 8;

// Daubechies extremal-phase db6 scaling (reconstruction low-pass) filter,
// obtained by spectral factorisation of P(y) = sum_k C(5 + k, k) y^k
// (Daubechies 1988); sum = sqrt(2), unit norm.
static const double kDb6RecLo[kF] = {
    0.11154074335010940,  0.49462389039845290,  0.75113390802109490,  0.31525035170919800,
    -0.22626469396543930, -0.12976686756726188, 0.09750160558732306,  0.02752286553030561,
    -0.03158203931748598, 0.00055384220116150,  0.00477725751094551,  -0.00107730108530848};

struct Filters {
    float dec_lo[kF], dec_hi[kF], rec_lo[kF], rec_hi[kF];
};

struct WaveletPlan {
    int levels = 0;
    int in_shape[kMaxLevels][3];
    int out_shape[kMaxLevels][3];
    int64_t det_off[kMaxLevels];   // offset of level l's 7 detail bands (l = 0 finest)
    int64_t ncoef = 0;
    Filters f;
    float2* T1 = nullptr;
    float2* T2 = nullptr;
    float2* A[2] = {nullptr, nullptr};
    int64_t t1_elems = 0, t2_elems = 0, a_elems = 0;
    int nimg = 0;
};

static int dwt_len(int n) { return (n + kF - 1) / 2; }

static int max_level(const int* shape) {
    int lv = 1 << 30;
    for (int i = 0; i < 3; ++i) {
        int l = shape[i] < kF - 1 ? 0 : (int)std::floor(std::log2((double)shape[i] / (kF - 1)));
        lv = std::min(lv, l);
    }
    return std::max(lv, 0);
}

tr_status wavelet_prepare(tr_plan* p) {
    WaveletPlan* w = new WaveletPlan();
    p->wav = w;
    w->levels = std::min(max_level(p->n), kMaxLevels);
    int cur[3] = {p->n[0], p->n[1], p->n[2]};
    for (int l = 0; l < w->levels; ++l) {
        for (int i = 0; i < 3; ++i) {
            w->in_shape[l][i] = cur[i];
            w->out_shape[l][i] = dwt_len(cur[i]);
            cur[i] = w->out_shape[l][i];
        }
    }
    // layout: cA_L, det_L, ..., det_1
    int64_t off = 0;
    if (w->levels > 0) {
        const int* s = w->out_shape[w->levels - 1];
        off = (int64_t)s[0] * s[1] * s[2];
    }
    for (int l = w->levels - 1; l >= 0; --l) {
        const int* s = w->out_shape[l];
        w->det_off[l] = off;
        off += 7LL * s[0] * s[1] * s[2];
    }
    w->ncoef = off;
    for (int j = 0; j < kF; ++j) {
        const double lo = kDb6RecLo[kF - 1 - j];                      // dec_lo = reversed rec_lo
        const double hi = ((j + 1) % 2 ? -1.0 : 1.0) * kDb6RecLo[j];  // dec_hi[j] = (-1)^(j+1) dec_lo[F-1-j]
        w->f.dec_lo[j] = (float)lo;
        w->f.dec_hi[j] = (float)hi;
    }
    for (int j = 0; j < kF; ++j) {
        w->f.rec_lo[j] = w->f.dec_lo[kF - 1 - j];
        w->f.rec_hi[j] = w->f.dec_hi[kF - 1 - j];
    }
    return TR_OK;
}

void wavelet_info(const tr_plan* p, int32_t* levels, int64_t* coeffs) {
    if (levels) *levels = p->wav ? p->wav->levels : 0;
    if (coeffs) *coeffs = p->wav ? p->wav->ncoef : 0;
}

void wavelet_destroy(tr_plan* p) {
    if (!p->wav) return;
    cudaFree(p->wav->T1);
    cudaFree(p->wav->T2);
    cudaFree(p->wav->A[0]);
    cudaFree(p->wav->A[1]);
    delete p->wav;
    p->wav = nullptr;
}

static tr_status ensure_wavelet_buffers(tr_plan* p, int nimg) {
    WaveletPlan* w = p->wav;
    if (w->nimg >= nimg && w->T1) return TR_OK;
    cudaFree(w->T1);
    cudaFree(w->T2);
    cudaFree(w->A[0]);
    cudaFree(w->A[1]);
    w->T1 = w->T2 = w->A[0] = w->A[1] = nullptr;
    int64_t t1 = 0, t2 = 0, a = 0;
    for (int l = 0; l < w->levels; ++l) {
        const int* si = w->in_shape[l];
        const int* so = w->out_shape[l];
        t1 = std::max<int64_t>(t1, 2LL * so[0] * si[1] * si[2]);
        t2 = std::max<int64_t>(t2, 4LL * so[0] * so[1] * si[2]);
        a = std::max<int64_t>(a, (int64_t)so[0] * so[1] * so[2]);
        a = std::max<int64_t>(a, (int64_t)si[0] * si[1] * si[2]);
    }
    w->t1_elems = t1 * nimg;
    w->t2_elems = t2 * nimg;
    w->a_elems = a * nimg;
    TR_CUDA(cudaMalloc(&w->T1, w->t1_elems * sizeof(float2)));
    TR_CUDA(cudaMalloc(&w->T2, w->t2_elems * sizeof(float2)));
    TR_CUDA(cudaMalloc(&w->A[0], w->a_elems * sizeof(float2)));
    TR_CUDA(cudaMalloc(&w->A[1], w->a_elems * sizeof(float2)));
    p->workspace_bytes += (w->t1_elems + w->t2_elems + 2 * w->a_elems) * (int64_t)sizeof(float2);
    w->nimg = nimg;
    return TR_OK;
}

// ------------------------------------------------------------------ analysis
// in viewed as [P][n][Q] -> out [P][2][no][Q] (band 0 = low, 1 = high)
__global__ void k_dwt_pass(const float2* __restrict__ in, float2* __restrict__ out, int64_t P, int n, int64_t Q,
                           int no, Filters f) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = P * no * Q;
    if (t >= total) return;
    const int64_t q = t % Q;
    const int64_t r = t / Q;
    const int o = (int)(r % no);
    const int64_t pp = r / no;
    const float2* src = in + pp * n * Q + q;
    float2 lo = make_float2(0.f, 0.f), hi = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kF; ++j) {
        const int i = 2 * o + 1 - j;
        if (i < 0 || i >= n) continue;
        const float2 v = src[(int64_t)i * Q];
        lo.x += f.dec_lo[j] * v.x;
        lo.y += f.dec_lo[j] * v.y;
        hi.x += f.dec_hi[j] * v.x;
        hi.y += f.dec_hi[j] * v.y;
    }
    float2* dst = out + (pp * 2) * no * Q + (int64_t)o * Q + q;
    dst[0] = lo;
    dst[(int64_t)no * Q] = hi;
}

// Last (x) pass of one level: T2 (img, bz, Zo, by, Yo, Xi) -> 8 bands.
// Detail bands (and cA at the coarsest level) update the dual in place:
//   p <- p + sigma c,  p <- p * min(1, lam / sqrt(|p|^2 + 1e-12))   (lam <= 0: p <- 0)
// Band aaa of a non-coarsest level goes to the next level's input buffer.
struct DwtLastArgs {
    const float2* in;
    int nimg, Zo, Yo, Xi, Xo;
    float2* next;      // (nimg, Zo, Yo, Xo) or null at the coarsest level
    float2* pw2;       // (nimg, ncoef)
    int64_t ncoef, det_off;
    int coarsest;
    float sigma, lam;
    Filters f;
};

__global__ void k_dwt_last(DwtLastArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t rows = (int64_t)a.nimg * 2 * a.Zo * 2 * a.Yo;
    if (t >= rows * a.Xo) return;
    const int x = (int)(t % a.Xo);
    int64_t r = t / a.Xo;
    const int y = (int)(r % a.Yo);
    r /= a.Yo;
    const int by = (int)(r % 2);
    r /= 2;
    const int z = (int)(r % a.Zo);
    r /= a.Zo;
    const int bz = (int)(r % 2);
    const int64_t img = r / 2;
    const float2* src = a.in + (t / a.Xo) * a.Xi;
    float2 c[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
    for (int j = 0; j < kF; ++j) {
        const int i = 2 * x + 1 - j;
        if (i < 0 || i >= a.Xi) continue;
        const float2 v = src[i];
        c[0].x += a.f.dec_lo[j] * v.x;
        c[0].y += a.f.dec_lo[j] * v.y;
        c[1].x += a.f.dec_hi[j] * v.x;
        c[1].y += a.f.dec_hi[j] * v.y;
    }
    const int64_t sub = (int64_t)a.Zo * a.Yo * a.Xo;
    const int64_t pos = ((int64_t)z * a.Yo + y) * a.Xo + x;
#pragma unroll
    for (int bx = 0; bx < 2; ++bx) {
        const int band = bz * 4 + by * 2 + bx;
        float2* slot;
        if (band == 0) {
            if (!a.coarsest) {
                a.next[img * sub + pos] = c[bx];
                continue;
            }
            slot = a.pw2 + img * a.ncoef + pos;            // cA
        } else {
            slot = a.pw2 + img * a.ncoef + a.det_off + (int64_t)(band - 1) * sub + pos;
        }
        if (a.lam <= 0.f) {
            *slot = make_float2(0.f, 0.f);
            continue;
        }
        float2 pv = *slot;
        pv.x += a.sigma * c[bx].x;
        pv.y += a.sigma * c[bx].y;
        const float mag = sqrtf(pv.x * pv.x + pv.y * pv.y + 1e-12f);
        const float s = fminf(a.lam / mag, 1.0f);
        *slot = make_float2(pv.x * s, pv.y * s);
    }
}

// ------------------------------------------------------------------ synthesis
// First (x) pass of one level: 8 bands -> T2 (img, bz, Zo, by, Yo, Xi).
struct IdwtFirstArgs {
    const float2* approx;  // (nimg, Zo, Yo, Xo): band aaa
    const float2* pw2;     // (nimg, ncoef)
    int64_t ncoef, det_off;
    int nimg, Zo, Yo, Xo, Xi;
    float2* out;
    Filters f;
};

__global__ void k_idwt_first(IdwtFirstArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t rows = (int64_t)a.nimg * 2 * a.Zo * 2 * a.Yo;
    if (t >= rows * a.Xi) return;
    const int x = (int)(t % a.Xi);
    int64_t r = t / a.Xi;
    const int y = (int)(r % a.Yo);
    r /= a.Yo;
    const int by = (int)(r % 2);
    r /= 2;
    const int z = (int)(r % a.Zo);
    r /= a.Zo;
    const int bz = (int)(r % 2);
    const int64_t img = r / 2;
    const int64_t sub = (int64_t)a.Zo * a.Yo * a.Xo;
    const int64_t rowpos = ((int64_t)z * a.Yo + y) * a.Xo;
    const float2* lo;
    const int bl = bz * 4 + by * 2;
    if (bl == 0) lo = a.approx + img * sub + rowpos;
    else lo = a.pw2 + img * a.ncoef + a.det_off + (int64_t)(bl - 1) * sub + rowpos;
    const float2* hi = a.pw2 + img * a.ncoef + a.det_off + (int64_t)(bl + 1 - 1) * sub + rowpos;
    const int i0 = x / 2 + kF / 2 - 1;
    const int par = x & 1;
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kF / 2; ++j) {
        const int i = i0 - j;
        if (i < 0 || i >= a.Xo) continue;
        const float gl = a.f.rec_lo[2 * j + par], gh = a.f.rec_hi[2 * j + par];
        const float2 u = lo[i], v = hi[i];
        s.x += gl * u.x + gh * v.x;
        s.y += gl * u.y + gh * v.y;
    }
    a.out[t] = s;
}

// Generic synthesis along the middle axis of [P][2][no][Q] -> [P][ni][Q].
__global__ void k_idwt_pass(const float2* __restrict__ in, float2* __restrict__ out, int64_t P, int no, int64_t Q,
                            int ni, Filters f) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P * ni * Q) return;
    const int64_t q = t % Q;
    const int64_t r = t / Q;
    const int o = (int)(r % ni);
    const int64_t pp = r / ni;
    const float2* lo = in + (pp * 2) * no * Q + q;
    const float2* hi = lo + (int64_t)no * Q;
    const int i0 = o / 2 + kF / 2 - 1;
    const int par = o & 1;
    float2 s = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < kF / 2; ++j) {
        const int i = i0 - j;
        if (i < 0 || i >= no) continue;
        const float gl = f.rec_lo[2 * j + par], gh = f.rec_hi[2 * j + par];
        const float2 u = lo[(int64_t)i * Q], v = hi[(int64_t)i * Q];
        s.x += gl * u.x + gh * v.x;
        s.y += gl * u.y + gh * v.y;
    }
    out[t] = s;
}

static unsigned nblk(int64_t n) { return (unsigned)((n + 255) / 256); }

tr_status wavelet_dual(tr_plan* p, const float2* u_bar, float2* p_w2, float sigma, float lam, cudaStream_t st) {
    WaveletPlan* w = p->wav;
    const int nimg = p->B * p->E;
    if (w->levels == 0) return fail(TR_ERR_UNSUPPORTED, "image too small for a db6 decomposition");
    TR_TRY(ensure_wavelet_buffers(p, nimg));
    const float2* cur = u_bar;
    for (int l = 0; l < w->levels; ++l) {
        const int* si = w->in_shape[l];
        const int* so = w->out_shape[l];
        // z
        int64_t P = nimg, Q = (int64_t)si[1] * si[2];
        k_dwt_pass<<<nblk(P * so[0] * Q), 256, 0, st>>>(cur, w->T1, P, si[0], Q, so[0], w->f);
        TR_CHECK_LAUNCH();
        // y: T1 [nimg*2*Zo][Yi][Xi]
        P = (int64_t)nimg * 2 * so[0];
        Q = si[2];
        k_dwt_pass<<<nblk(P * so[1] * Q), 256, 0, st>>>(w->T1, w->T2, P, si[1], Q, so[1], w->f);
        TR_CHECK_LAUNCH();
        // x + dual update
        DwtLastArgs a;
        a.in = w->T2;
        a.nimg = nimg;
        a.Zo = so[0];
        a.Yo = so[1];
        a.Xi = si[2];
        a.Xo = so[2];
        a.coarsest = (l == w->levels - 1);
        a.next = a.coarsest ? nullptr : w->A[l & 1];
        a.pw2 = p_w2;
        a.ncoef = w->ncoef;
        a.det_off = w->det_off[l];
        a.sigma = sigma;
        a.lam = lam;
        a.f = w->f;
        const int64_t n = (int64_t)nimg * 4 * so[0] * so[1] * so[2];
        k_dwt_last<<<nblk(n), 256, 0, st>>>(a);
        TR_CHECK_LAUNCH();
        cur = a.next;
    }
    return TR_OK;
}

tr_status wavelet_adjoint(tr_plan* p, const float2* p_w2, float2* out, cudaStream_t st) {
    WaveletPlan* w = p->wav;
    const int nimg = p->B * p->E;
    if (w->levels == 0) return fail(TR_ERR_UNSUPPORTED, "image too small for a db6 decomposition");
    TR_TRY(ensure_wavelet_buffers(p, nimg));
    // approximation of the coarsest level lives in p_w2 (cA); copy it to A[0]
    const int Lc = w->levels - 1;
    const int* sc = w->out_shape[Lc];
    const int64_t nca = (int64_t)sc[0] * sc[1] * sc[2];
    TR_CUDA(cudaMemcpy2DAsync(w->A[0], nca * sizeof(float2), p_w2, w->ncoef * sizeof(float2), nca * sizeof(float2),
                              nimg, cudaMemcpyDeviceToDevice, st));
    int ai = 0;
    for (int l = Lc; l >= 0; --l) {
        const int* si = w->in_shape[l];
        const int* so = w->out_shape[l];
        IdwtFirstArgs a;
        a.approx = w->A[ai];
        a.pw2 = p_w2;
        a.ncoef = w->ncoef;
        a.det_off = w->det_off[l];
        a.nimg = nimg;
        a.Zo = so[0];
        a.Yo = so[1];
        a.Xo = so[2];
        a.Xi = si[2];
        a.out = w->T2;
        a.f = w->f;
        k_idwt_first<<<nblk((int64_t)nimg * 4 * so[0] * so[1] * si[2]), 256, 0, st>>>(a);
        TR_CHECK_LAUNCH();
        // y: T2 [nimg*2*Zo][2][Yo][Xi] -> T1 [nimg*2*Zo][Yi][Xi]
        int64_t P = (int64_t)nimg * 2 * so[0], Q = si[2];
        k_idwt_pass<<<nblk(P * si[1] * Q), 256, 0, st>>>(w->T2, w->T1, P, so[1], Q, si[1], w->f);
        TR_CHECK_LAUNCH();
        // z: T1 [nimg][2][Zo][Yi*Xi] -> (nimg, Zi, Yi, Xi)
        P = nimg;
        Q = (int64_t)si[1] * si[2];
        float2* dst = (l == 0) ? out : w->A[ai ^ 1];
        k_idwt_pass<<<nblk(P * si[0] * Q), 256, 0, st>>>(w->T1, dst, P, so[0], Q, si[0], w->f);
        TR_CHECK_LAUNCH();
        ai ^= 1;
    }
    return TR_OK;
}

}  // namespace tr

using namespace tr;

// W2 analysis alone: the dual update of wavelet_dual with a zero dual, unit step
// and an inactive projection (p = 0 + 1 c, scale min(1, FLT_MAX / |c|) = 1) is
// the coefficient tree itself, bit for bit.
extern "C" tr_status tr_wavelet_forward(tr_plan* p, const void* images, void* coeffs, void* stream) {
    if (!p || !images || !coeffs) return fail(TR_ERR_INVALID_ARG, "tr_wavelet_forward: null argument");
    if (!p->wav || p->wav->levels == 0)
        return fail(TR_ERR_UNSUPPORTED, "image too small for a db6 decomposition");
    DeviceGuard g(p->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = (size_t)p->B * p->E * p->wav->ncoef * sizeof(float2);
    TR_CUDA(cudaMemsetAsync(coeffs, 0, bytes, st));
    return wavelet_dual(p, (const float2*)images, (float2*)coeffs, 1.0f, FLT_MAX, st);
}

extern "C" tr_status tr_wavelet_adjoint(tr_plan* p, const void* coeffs, void* images, void* stream) {
    if (!p || !images || !coeffs) return fail(TR_ERR_INVALID_ARG, "tr_wavelet_adjoint: null argument");
    if (!p->wav || p->wav->levels == 0)
        return fail(TR_ERR_UNSUPPORTED, "image too small for a db6 decomposition");
    DeviceGuard g(p->device);
    return wavelet_adjoint(p, (const float2*)coeffs, (float2*)images, (cudaStream_t)stream);
}
