// PDHG iterations for TVM / TVME / TVMW on one B200.
//
// One iteration (the reference's order, single device, every ghost a global edge):
//   1. data dual   q_b <- (q_b + sigma (F_b(u_bar S) - y_b)) / (1 + sigma)      [NUFFT forward, fused]
//   2. TV duals    one pass over (B, E, Z, Y, X): motion (L1 or L2 over echoes),
//                  TVME echo-spatial isotropic TV, TVMW db1 echo wavelet       [k_dual]
//      TVMW       db6 spatial wavelet dual with the L-inf projection         [tr_wavelet.cu]
//   3. data grad   g_b = sum_c conj(S_c) F_b^H(dcf q_b)                        [NUFFT adjoint, fused]
//      TVMW       w2adj = waverec3(p_w2)
//   4. primal      u <- u - tau(...), u_bar <- 2 u_new - u_old, FP64 partial
//                  sums of the stopping tolerance                              [k_primal]
//   5. tolerance   fixed-order FP64 reduction of the partial sums             [k_tol_finalize]
//
// Reference: tvm.py:227-380, tvme.py:208-482, tvmw.py:385-685 (iteration),
// tvm.py:406-472, tvme.py:512-557, tvmw.py:716-773 (tolerance and stop).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "tr_internal.cuh"

namespace tr {

// Text of the device error word's bits (kDevErr*).
static std::string device_error_text(int bits) {
    std::string s;
    if (bits & kDevErrTmaWait) s += "a bounded device wait expired";
    if (bits & kDevErrCluster) s += std::string(s.empty() ? "" : " and ") + "a cluster kernel ran without its cluster";
    if (s.empty()) s = "a device-side check failed";
    return s + " (error bits " + std::to_string(bits) + ")";
}

struct PdhgGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    tr_pdhg_state state;
    tr_pdhg_params params;
    cudaStream_t stream = nullptr;
};

void pdhg_destroy(tr_plan* p) {
    if (!p->graph) return;
    if (p->graph->exec) cudaGraphExecDestroy(p->graph->exec);
    if (p->graph->graph) cudaGraphDestroy(p->graph->graph);
    delete p->graph;
    p->graph = nullptr;
}

struct PdArgs {
    const float2* ubar;
    float2* u;
    float2* ubar_out;
    const float2* g;
    const float2* w2adj;
    float2* pm;
    float2* pex;
    float2* pey;
    float2* pez;
    float2* pw1;
    int alg, l2;
    int B, E, Z, Y, X;
    int Bg, b0;                 // bins of the whole problem; global index of local bin 0
    const float2* ubar_next;    // (E, N) u_bar of global bin b0 + B (another rank's), or null
    const float2* pm_prev;      // (E, N) p_m of global bin b0 - 1 (another rank's), or null
    int64_t N;
    float sigma, tau, lam_m, lam_e, lam_w1;
    double* partials;
};

__device__ __forceinline__ float cabsf(float2 v) { return sqrtf(v.x * v.x + v.y * v.y); }

// ------------------------------------------------------------------ duals
// EC > 0: the echo count as a compile-time constant (the echo loops unroll, so
// every echo's loads are in flight together); EC = 0: any echo count.
template <int EC>
__global__ void __launch_bounds__(256) k_dual(PdArgs a) {
    const int E = EC > 0 ? EC : a.E;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)a.B * a.N) return;
    const int b = (int)(t / a.N);
    const int64_t v = t - (int64_t)b * a.N;
    const int YX = a.Y * a.X;
    const int z = (int)(v / YX);
    const int rem = (int)(v - (int64_t)z * YX);
    const int y = rem / a.X;
    const int x = rem - y * a.X;
    const int64_t EN = (int64_t)E * a.N;
    const float2* ub = a.ubar + (int64_t)b * EN;
    // u_bar of the next global bin: local, the halo from the next rank, or none at the global end
    const float2* ubn = (b + 1 < a.B) ? ub + EN : ((a.b0 + b + 1 < a.Bg) ? a.ubar_next : nullptr);
    const float sig = a.sigma;
    // p / max(1, |p| / lambda) as p * (1 / max(1, |p| (1 / lambda))): one division per
    // projection instead of one per component and per ratio (the kernel is issue-bound)
    const float ilam_m = 1.0f / a.lam_m, ilam_e = 1.0f / a.lam_e;
    float s2 = 0.f;
#pragma unroll (EC > 0 ? EC : 1)
    for (int e = 0; e < E; ++e) {
        const int64_t o = (int64_t)b * EN + (int64_t)e * a.N + v;
        const float2 u0 = ub[(int64_t)e * a.N + v];
        // motion: p_m += sigma (u_bar[b+1] - u_bar[b]) (0 at the last bin)
        float2 dm = make_float2(0.f, 0.f);
        if (ubn) dm = csub(ubn[(int64_t)e * a.N + v], u0);
        float2 pm = a.pm[o];
        pm = make_float2(pm.x + sig * dm.x, pm.y + sig * dm.y);
        if (!a.l2) {
            pm = cscale(pm, 1.0f / fmaxf(1.0f, cabsf(pm) * ilam_m));
        } else {
            const float m = cabsf(pm);
            s2 += m * m;
        }
        a.pm[o] = pm;
        if (a.alg == TR_ALG_TVME) {
            float2 gx = make_float2(0.f, 0.f), gy = gx, gz = gx;
            if (e + 1 < E) {
                const float2* u_e = ub + (int64_t)e * a.N;
                const float2* u_n = u_e + a.N;
                const float2 d0 = csub(u_n[v], u_e[v]);
                if (x + 1 < a.X) gx = csub(csub(u_n[v + 1], u_e[v + 1]), d0);
                if (y + 1 < a.Y) gy = csub(csub(u_n[v + a.X], u_e[v + a.X]), d0);
                if (z + 1 < a.Z) gz = csub(csub(u_n[v + YX], u_e[v + YX]), d0);
            }
            float2 px = a.pex[o], py = a.pey[o], pz = a.pez[o];
            px = make_float2(px.x + sig * gx.x, px.y + sig * gx.y);
            py = make_float2(py.x + sig * gy.x, py.y + sig * gy.y);
            pz = make_float2(pz.x + sig * gz.x, pz.y + sig * gz.y);
            // (|px|^2 + |py|^2 + |pz|^2)^(1/2) from the squared components
            const float mag2 = (px.x * px.x + px.y * px.y) + (py.x * py.x + py.y * py.y) + (pz.x * pz.x + pz.y * pz.y);
            const float inv = 1.0f / fmaxf(1.0f, sqrtf(mag2) * ilam_e);
            a.pex[o] = cscale(px, inv);
            a.pey[o] = cscale(py, inv);
            a.pez[o] = cscale(pz, inv);
        } else if (a.alg == TR_ALG_TVMW) {
            // db1 along echo: even e: (u_e + u_{e+1})/sqrt2 ; odd e: (u_e - u_{e-1})/sqrt2
            const float s = 0.70710678118654752f;
            float2 w;
            if ((e & 1) == 0) {
                float2 x1 = (e + 1 < E) ? ub[(int64_t)(e + 1) * a.N + v] : make_float2(0.f, 0.f);
                w = cscale(cadd(u0, x1), s);
            } else {
                const float2 xm = ub[(int64_t)(e - 1) * a.N + v];
                w = cscale(cadd(make_float2(-xm.x, -xm.y), u0), s);
            }
            float2 pw = a.pw1[o];
            pw = make_float2(pw.x + sig * w.x, pw.y + sig * w.y);
            if (a.lam_w1 > 0.f) {
                pw = cscale(pw, 1.0f / fmaxf(1.0f, cabsf(pw) / a.lam_w1));
            } else {
                pw = make_float2(0.f, 0.f);
            }
            a.pw1[o] = pw;
        }
    }
    if (a.l2) {
        const float inv = 1.0f / fmaxf(1.0f, sqrtf(s2) * ilam_m);
#pragma unroll (EC > 0 ? EC : 1)
        for (int e = 0; e < E; ++e) {
            const int64_t o = (int64_t)b * EN + (int64_t)e * a.N + v;
            a.pm[o] = cscale(a.pm[o], inv);
        }
    }
}

// Exact transpose of the zero-last-row forward difference along one axis:
// d[i] = -p[i] (i < n-1) + p[i-1] (i >= 1).
__device__ __forceinline__ float2 back_diff(const float2* p, int64_t v, int64_t stride, int i, int n) {
    float2 d = make_float2(0.f, 0.f);
    if (i >= 1) d = p[v - stride];
    if (i < n - 1) d = csub(d, p[v]);
    return d;
}

__device__ __forceinline__ void block_reduce_partials(double num, double den, double* partials) {
    __shared__ double sn[8], sd[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        num += __shfl_down_sync(0xffffffffu, num, off);
        den += __shfl_down_sync(0xffffffffu, den, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sn[warp] = num;
        sd[warp] = den;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += sn[w];
            b += sd[w];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
    }
}

// ------------------------------------------------------------------ primal + extrapolation + tolerance
__global__ void __launch_bounds__(256) k_primal(PdArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double num = 0.0, den = 0.0;
    if (t < (int64_t)a.B * a.N) {
        const int b = (int)(t / a.N);
        const int64_t v = t - (int64_t)b * a.N;
        const int YX = a.Y * a.X;
        const int z = (int)(v / YX);
        const int rem = (int)(v - (int64_t)z * YX);
        const int y = rem / a.X;
        const int x = rem - y * a.X;
        const int64_t EN = (int64_t)a.E * a.N;
        const float tau = a.tau;
        const int gb = a.b0 + b;              // global bin
        float2 divprev = make_float2(0.f, 0.f);
        for (int e = 0; e < a.E; ++e) {
            const int64_t o = (int64_t)b * EN + (int64_t)e * a.N + v;
            const float2 uo = a.u[o];
            const float2 g = a.g[o];
            // p_m of the previous global bin: local, or the halo from the previous rank
            float2 pprev = make_float2(0.f, 0.f);
            if (gb > 0) pprev = (b > 0) ? a.pm[o - EN] : a.pm_prev[(int64_t)e * a.N + v];
            float2 un;
            if (a.alg == TR_ALG_TVME) {
                // divp_m = D_m^T p_m  (tvme.py:421-437)
                float2 dm = make_float2(0.f, 0.f);
                if (a.Bg > 1) {
                    if (gb == 0) dm = make_float2(-a.pm[o].x, -a.pm[o].y);
                    else if (gb == a.Bg - 1) dm = pprev;
                    else dm = csub(pprev, a.pm[o]);
                }
                // divp = dxb(p_ex) + dyb(p_ey) + dzb(p_ez) at (b, e)
                const float2 dx = back_diff(a.pex + (o - v), v, 1, x, a.X);
                const float2 dy = back_diff(a.pey + (o - v), v, a.X, y, a.Y);
                const float2 dz = back_diff(a.pez + (o - v), v, YX, z, a.Z);
                const float2 divc = cadd(cadd(dx, dy), dz);
                // divp_e = D_e^T divp  (tvme.py:361-363, :444-454)
                float2 de;
                if (e == 0) de = make_float2(-divc.x, -divc.y);
                else if (e == a.E - 1) de = divprev;
                else de = csub(divprev, divc);
                divprev = divc;
                un = make_float2(uo.x - tau * dm.x, uo.y - tau * dm.y);
                un = make_float2(un.x - tau * de.x, un.y - tau * de.y);
                un = make_float2(un.x - tau * g.x, un.y - tau * g.y);
            } else if (a.alg == TR_ALG_TVM) {
                // divergence = p[b] - p[b-1] with the reference's edges (tvm.py:342-357)
                float2 dv;
                if (a.Bg == 1) dv = make_float2(0.f, 0.f);
                else if (gb == 0) dv = a.pm[o];
                else if (gb == a.Bg - 1) dv = make_float2(-pprev.x, -pprev.y);
                else dv = csub(a.pm[o], pprev);
                const float2 r = csub(g, dv);
                un = make_float2(uo.x + (-tau) * r.x, uo.y + (-tau) * r.y);
            } else {
                // TVMW: u_tmp -= tau (g - divp_m + divp_w1 + divp_w2)  (tvmw.py:662-681)
                float2 dvm = (gb == 0) ? a.pm[o] : csub(a.pm[o], pprev);
                const float s = 0.70710678118654752f;
                float2 w1;
                if ((e & 1) == 0) {
                    const float2 dn = (e + 1 < a.E) ? a.pw1[o + a.N] : make_float2(0.f, 0.f);
                    w1 = cscale(csub(a.pw1[o], dn), s);
                } else {
                    w1 = cscale(cadd(a.pw1[o - a.N], a.pw1[o]), s);
                }
                const float2 r = cadd(cadd(csub(g, dvm), w1), a.w2adj[o]);
                un = make_float2(uo.x - tau * r.x, uo.y - tau * r.y);
            }
            const float2 ubn = make_float2(2.0f * un.x - uo.x, 2.0f * un.y - uo.y);
            a.u[o] = un;
            if (a.alg == TR_ALG_TVMW) {
                // tolerance on u_bar: ||u_bar_prev - u_bar_new|| / ||u_bar_prev|| (tvmw.py:721-769)
                const float2 up = a.ubar[o];
                const double ddx = (double)up.x - (double)ubn.x, ddy = (double)up.y - (double)ubn.y;
                num += ddx * ddx + ddy * ddy;
                den += (double)up.x * up.x + (double)up.y * up.y;
            } else {
                // tolerance on u: ||u_new - u_old|| / ||u_new|| (tvme.py:518-551)
                const double ddx = (double)un.x - (double)uo.x, ddy = (double)un.y - (double)uo.y;
                num += ddx * ddx + ddy * ddy;
                den += (double)un.x * un.x + (double)un.y * un.y;
            }
            a.ubar_out[o] = ubn;
        }
    }
    block_reduce_partials(num, den, a.partials);
}

// One CTA sums the n (num, den) pairs in a fixed order: thread t takes pairs
// t, t + T, t + 2T, ... into four accumulators by turn (four 16-byte loads in
// flight per thread), adds them pairwise, and a fixed tree combines the
// threads.  Launched with kTolThreads threads; 196,608 pairs (TVME-256, six
// bins) take about 20 us instead of the 0.37 ms of one accumulator per thread
// on 256 threads.
constexpr int kTolThreads = 1024;
__global__ void __launch_bounds__(kTolThreads) k_tol_finalize(const double* __restrict__ partials, int n,
                                                              double* out) {
    __shared__ double sn[kTolThreads], sd[kTolThreads];
    const double2* p2 = reinterpret_cast<const double2*>(partials);     // cudaMalloc'd: 16-byte aligned
    double a[4] = {0.0, 0.0, 0.0, 0.0}, b[4] = {0.0, 0.0, 0.0, 0.0};
    int i = threadIdx.x;
    for (; i + 3 * kTolThreads < n; i += 4 * kTolThreads) {
        double2 v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = p2[i + k * kTolThreads];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[k] += v[k].x;
            b[k] += v[k].y;
        }
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {             // fewer than four strides remain
        if (i < n) {
            const double2 v = p2[i];
            a[k] += v.x;
            b[k] += v.y;
        }
        i += kTolThreads;
    }
    sn[threadIdx.x] = (a[0] + a[1]) + (a[2] + a[3]);
    sd[threadIdx.x] = (b[0] + b[1]) + (b[2] + b[3]);
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

// ------------------------------------------------------------------ driver
static tr_status validate(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q) {
    if (!p || !s || !q) return fail(TR_ERR_INVALID_ARG, "tr_pdhg_run: null argument");
    if (!p->maps) return fail(TR_ERR_INVALID_ARG, "coil maps not set (tr_plan_set_maps)");
    if (!s->u || !s->u_bar || !s->p_m || !s->q || !s->y || !s->g)
        return fail(TR_ERR_INVALID_ARG, "state u, u_bar, p_m, q, y and g are required");
    if (q->algorithm == TR_ALG_TVME && (!s->p_ex || !s->p_ey || !s->p_ez))
        return fail(TR_ERR_INVALID_ARG, "TVME needs p_ex, p_ey, p_ez");
    if (q->algorithm == TR_ALG_TVMW && (!s->p_w1 || !s->p_w2 || !s->w2adj))
        return fail(TR_ERR_INVALID_ARG, "TVMW needs p_w1, p_w2, w2adj");
    if (q->algorithm < 0 || q->algorithm > 2) return fail(TR_ERR_INVALID_ARG, "unknown algorithm");
    if (!(q->sigma > 0.f) || !(q->tau > 0.f)) return fail(TR_ERR_INVALID_ARG, "sigma and tau must be positive");
    if (!(q->sigma_data >= 0.f)) return fail(TR_ERR_INVALID_ARG, "sigma_data must be >= 0 (0: use sigma)");
    return TR_OK;
}

// Local bins [0, B) of the plan sit at global bins [b0, b0 + B) of Bg; the
// halos carry the neighbouring ranks' edge bins (null where this plan holds the
// global first / last bin).
struct ShardView {
    int Bg = 0, b0 = 0;
    const float2* ubar_next = nullptr;
    const float2* pm_prev = nullptr;
};

static PdArgs make_args(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, const ShardView& sh) {
    PdArgs a;
    memset(&a, 0, sizeof(a));
    a.ubar = (const float2*)s->u_bar;
    a.u = (float2*)s->u;
    a.ubar_out = (float2*)s->u_bar;
    a.g = (const float2*)s->g;
    a.w2adj = (const float2*)s->w2adj;
    a.pm = (float2*)s->p_m;
    a.pex = (float2*)s->p_ex;
    a.pey = (float2*)s->p_ey;
    a.pez = (float2*)s->p_ez;
    a.pw1 = (float2*)s->p_w1;
    a.alg = q->algorithm;
    a.l2 = q->l2_coupling;
    a.B = p->B;
    a.E = p->E;
    a.Z = p->n[0];
    a.Y = p->n[1];
    a.X = p->n[2];
    a.Bg = sh.Bg > 0 ? sh.Bg : p->B;
    a.b0 = sh.b0;
    a.ubar_next = sh.ubar_next;
    a.pm_prev = sh.pm_prev;
    a.N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    a.sigma = q->sigma;
    a.tau = q->tau;
    a.lam_m = q->lam_m;
    a.lam_e = q->lam_e;
    a.lam_w1 = q->lam_w1;
    return a;
}

// Phase 1: every dual update and the data gradient (reads u_bar, u_bar_next).
// Phase 1 is enqueued in two parts: `local` (the TVMW spatial-wavelet dual and
// the data dual; they read only this plan's u_bar) and `halo` (the TV / W1 duals,
// which read u_bar_next, and the data gradient).  A sharded caller posts the
// u_bar halo, enqueues the local part while it travels, then the halo part.
static tr_status enqueue_phase1_local(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, cudaStream_t st) {
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    const int64_t EN = (int64_t)p->E * N;
    const int ncol = p->E * p->C;
    float2* ubar = (float2*)s->u_bar;
    float2* qd = (float2*)s->q;
    const float2* y = (const float2*)s->y;
    // TVMW: the spatial-wavelet dual reads u_bar before anything changes it
    if (q->algorithm == TR_ALG_TVMW)
        TR_TRY(wavelet_dual(p, ubar, (float2*)s->p_w2, q->sigma, q->lam_w2, st));
    // 1. data dual (its own step when the caller gives one)
    const float sigma_data = q->sigma_data > 0.f ? q->sigma_data : q->sigma;
    for (int b = 0; b < p->B; ++b) {
        const int64_t off = p->bins[b].offset * ncol;
        TR_TRY(nufft_forward_cols(p, b, ubar + (int64_t)b * EN, N, p->E, p->maps, p->C, kInterpDualProx, sigma_data,
                                  y + off, qd + off, st));
    }
    return TR_OK;
}

static tr_status enqueue_phase1_halo(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, const ShardView& sh,
                                     cudaStream_t st) {
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    const int64_t EN = (int64_t)p->E * N;
    const int ncol = p->E * p->C;
    float2* qd = (float2*)s->q;
    float2* g = (float2*)s->g;
    // 2. TV / W1 duals
    PdArgs a = make_args(p, s, q, sh);
    const unsigned blocks = (unsigned)(((int64_t)p->B * N + 255) / 256);
    switch (p->E) {
        case 1: k_dual<1><<<blocks, 256, 0, st>>>(a); break;
        case 2: k_dual<2><<<blocks, 256, 0, st>>>(a); break;
        case 3: k_dual<3><<<blocks, 256, 0, st>>>(a); break;
        case 4: k_dual<4><<<blocks, 256, 0, st>>>(a); break;
        case 6: k_dual<6><<<blocks, 256, 0, st>>>(a); break;
        case 8: k_dual<8><<<blocks, 256, 0, st>>>(a); break;
        default: k_dual<0><<<blocks, 256, 0, st>>>(a); break;
    }
    TR_CHECK_LAUNCH();
    // 3. coil-combined, density-weighted adjoint
    for (int b = 0; b < p->B; ++b) {
        const int64_t off = p->bins[b].offset * ncol;
        TR_TRY(nufft_adjoint_cols(p, b, qd + off, p->E, p->maps, p->C, true, g + (int64_t)b * EN, N, st));
    }
    if (q->algorithm == TR_ALG_TVMW) TR_TRY(wavelet_adjoint(p, (const float2*)s->p_w2, (float2*)s->w2adj, st));
    return TR_OK;
}

static tr_status enqueue_phase1(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, const ShardView& sh,
                                cudaStream_t st) {
    TR_TRY(enqueue_phase1_local(p, s, q, st));
    return enqueue_phase1_halo(p, s, q, sh, st);
}

// Phase 2: primal update, extrapolation and the FP64 tolerance sums of the
// local bins into sums_out[2] (device memory); reads p_m and p_m_prev.
static tr_status enqueue_phase2(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, const ShardView& sh,
                                double* sums_out, cudaStream_t st) {
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    const unsigned blocks = (unsigned)(((int64_t)p->B * N + 255) / 256);
    if (!p->partials || p->npartials < (int)blocks) {
        cudaFree(p->partials);
        p->partials = nullptr;
        TR_CUDA(cudaMalloc(&p->partials, (size_t)blocks * 2 * sizeof(double)));
        p->npartials = (int)blocks;
    }
    PdArgs a = make_args(p, s, q, sh);
    a.partials = p->partials;
    k_primal<<<blocks, 256, 0, st>>>(a);
    TR_CHECK_LAUNCH();
    k_tol_finalize<<<1, kTolThreads, 0, st>>>(p->partials, (int)blocks, sums_out);
    TR_CHECK_LAUNCH();
    return TR_OK;
}

static tr_status enqueue_iteration(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, cudaStream_t st) {
    const ShardView whole;
    TR_TRY(enqueue_phase1(p, s, q, whole, st));
    TR_TRY(enqueue_phase2(p, s, q, whole, p->tol_dev, st));
    TR_CUDA(cudaMemcpyAsync(p->tol_host, p->tol_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    TR_CUDA(cudaMemcpyAsync(p->err_host, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    return TR_OK;
}

static double tolerance_from(const tr_pdhg_params* q, double num, double den) {
    if (q->algorithm == TR_ALG_TVMW) {
        if (std::isfinite(num) && std::isfinite(den))
            return std::sqrt(std::max(num, 0.0)) / std::max(std::sqrt(std::max(den, 0.0)), 1e-12);
        return INFINITY;
    }
    if (std::isfinite(num) && std::isfinite(den) && den > 0.0) return std::sqrt(std::max(num, 0.0)) / std::sqrt(den);
    return INFINITY;
}

static bool same_config(const PdhgGraph* g, const tr_pdhg_state* s, const tr_pdhg_params* q, cudaStream_t st) {
    return g && g->exec && g->stream == st && memcmp(&g->state, s, sizeof(*s)) == 0 &&
           memcmp(&g->params, q, sizeof(*q)) == 0;
}

static tr_status run_impl(tr_plan* p, const tr_pdhg_state* s, const tr_pdhg_params* q, int max_iters, double tol,
                          double* hist, int* done, cudaStream_t st) {
    TR_TRY(validate(p, s, q));
    int it = 0;
    for (; it < max_iters; ++it) {
        const bool use_graph = q->use_graph && it > 0;  // iteration 0 runs eagerly (allocates workspaces)
        if (use_graph) {
            if (!same_config(p->graph, s, q, st)) {
                pdhg_destroy(p);
                p->graph = new PdhgGraph();
                p->graph->state = *s;
                p->graph->params = *q;
                p->graph->stream = st;
                TR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                tr_status e = enqueue_iteration(p, s, q, st);
                cudaGraph_t graph = nullptr;
                cudaError_t ce = cudaStreamEndCapture(st, &graph);
                if (e != TR_OK) {
                    if (graph) cudaGraphDestroy(graph);
                    pdhg_destroy(p);
                    return e;
                }
                if (ce != cudaSuccess) {
                    pdhg_destroy(p);
                    return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
                }
                p->graph->graph = graph;
                TR_CUDA(cudaGraphInstantiate(&p->graph->exec, graph, 0));
            }
            TR_CUDA(cudaGraphLaunch(p->graph->exec, st));
        } else {
            TR_TRY(enqueue_iteration(p, s, q, st));
        }
        TR_CUDA(cudaStreamSynchronize(st));
        if (*p->err_host != 0) {
            const int bits = *p->err_host;
            *p->err_host = 0;
            cudaMemsetAsync(p->dev_err, 0, sizeof(int), st);
            if (done) *done = it;
            return fail(TR_ERR_TIMEOUT, device_error_text(bits) + " in iteration " + std::to_string(it) +
                                            "; results are invalid");
        }
        const double t = tolerance_from(q, p->tol_host[0], p->tol_host[1]);
        if (hist) hist[it] = t;
        if (!std::isfinite(p->tol_host[0]) || !std::isfinite(p->tol_host[1])) {
            if (done) *done = it + 1;
            return fail(TR_ERR_NONFINITE, "non-finite value in the tolerance reduction at iteration " +
                                              std::to_string(it));
        }
        if (t < tol) {
            ++it;
            break;
        }
    }
    if (done) *done = it;
    return TR_OK;
}

}  // namespace tr

using namespace tr;

extern "C" tr_status tr_pdhg_run(tr_plan* plan, const tr_pdhg_state* state, const tr_pdhg_params* params,
                                 int32_t max_iters, double tol, double* tol_history, int32_t* iters_done,
                                 void* stream) {
    if (!plan) return fail(TR_ERR_INVALID_ARG, "null plan");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != plan->device) cudaSetDevice(plan->device);
    int done = 0;
    tr_status s = run_impl(plan, state, params, max_iters, tol, tol_history, &done, (cudaStream_t)stream);
    if (iters_done) *iters_done = done;
    if (prev >= 0 && prev != plan->device) cudaSetDevice(prev);
    return s;
}

extern "C" tr_status tr_pdhg_phase(tr_plan* plan, const tr_pdhg_state* state, const tr_pdhg_params* params,
                                   const tr_pdhg_shard* shard, int32_t phase, double* tol_sums, void* stream) {
    if (!plan || !shard) return fail(TR_ERR_INVALID_ARG, "tr_pdhg_phase: null argument");
    TR_TRY(validate(plan, state, params));
    if (phase < 1 || phase > 4) return fail(TR_ERR_INVALID_ARG, "tr_pdhg_phase: phase must be 1, 2, 3 or 4");
    if (shard->bin_offset < 0 || shard->n_bins_global < shard->bin_offset + plan->B)
        return fail(TR_ERR_INVALID_ARG, "tr_pdhg_phase: n_bins_global must cover bin_offset + the plan's bins");
    const bool has_next = shard->bin_offset + plan->B < shard->n_bins_global;
    const bool has_prev = shard->bin_offset > 0;
    if ((phase == 1 || phase == 4) && has_next && !shard->u_bar_next)
        return fail(TR_ERR_INVALID_ARG, "tr_pdhg_phase: u_bar_next is required unless the plan holds the last bin");
    if (phase == 2 && has_prev && !shard->p_m_prev)
        return fail(TR_ERR_INVALID_ARG, "tr_pdhg_phase: p_m_prev is required unless the plan holds the first bin");
    if (phase == 2 && !tol_sums) return fail(TR_ERR_INVALID_ARG, "tr_pdhg_phase: tol_sums is required in phase 2");
    if (*plan->err_host != 0) {
        const int bits = *plan->err_host;
        *plan->err_host = 0;
        cudaMemsetAsync(plan->dev_err, 0, sizeof(int), (cudaStream_t)stream);
        return fail(TR_ERR_TIMEOUT, device_error_text(bits) + " in an earlier phase; results are invalid");
    }
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != plan->device) cudaSetDevice(plan->device);
    ShardView sh;
    sh.Bg = shard->n_bins_global;
    sh.b0 = shard->bin_offset;
    sh.ubar_next = has_next ? (const float2*)shard->u_bar_next : nullptr;
    sh.pm_prev = has_prev ? (const float2*)shard->p_m_prev : nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    tr_status rc;
    if (phase == 1) {
        rc = enqueue_phase1(plan, state, params, sh, st);
    } else if (phase == 3) {
        rc = enqueue_phase1_local(plan, state, params, st);
    } else if (phase == 4) {
        rc = enqueue_phase1_halo(plan, state, params, sh, st);
    } else {
        rc = enqueue_phase2(plan, state, params, sh, tol_sums, st);
        if (rc == TR_OK && cudaMemcpyAsync(plan->err_host, plan->dev_err, sizeof(int), cudaMemcpyDeviceToHost, st) !=
                               cudaSuccess)
            rc = fail(TR_ERR_CUDA, "tr_pdhg_phase: error-word copy failed");
    }
    if (prev >= 0 && prev != plan->device) cudaSetDevice(prev);
    return rc;
}

// ------------------------------------------------------------------ FP64 diagnostics
__global__ void k_norm2(const float2* __restrict__ x, int64_t n, double* partials) {
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = x[i];
        s += (double)v.x * v.x + (double)v.y * v.y;
    }
    block_reduce_partials(s, 0.0, partials);
}

__global__ void k_scale(float2* x, int64_t n, const double* nrm2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double inv = nrm2[0] > 0.0 ? 1.0 / sqrt(nrm2[0]) : 0.0;
    x[i] = make_float2((float)(x[i].x * inv), (float)(x[i].y * inv));
}

// Device scratch owned by one call, freed on every return path.
struct DevBuf {
    void* ptr = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (ptr) cudaFree(ptr);
    }
};

// ||x||^2 in FP64 into d2[0] (fixed-order: block partials, then one block).
static tr_status norm2_async(const float2* x, int64_t n, double* part, int nb, double* d2, cudaStream_t st) {
    k_norm2<<<nb, 256, 0, st>>>(x, n, part);
    TR_CHECK_LAUNCH();
    k_tol_finalize<<<1, kTolThreads, 0, st>>>(part, nb, d2);
    TR_CHECK_LAUNCH();
    return TR_OK;
}

// Power iteration on A^H W A with A = [F_b S_c] and W the density weights (the
// operator the PDHG data term sees; the reference has no such estimate).  The
// operator is block diagonal over (bin, echo) and every echo of a bin sees the
// same block, so one image per bin carries the whole spectrum: x is (B, Z, Y, X).
// Each step normalises x, applies the forward and density-weighted adjoint
// NUFFT over the C coil columns of every bin, and reads ||A^H W A x|| (FP64),
// which tends to the largest eigenvalue lambda; the norm returned is
// sqrt(lambda).
static tr_status power_impl(tr_plan* p, int n_iter, float2* x, double* norm_out, cudaStream_t st) {
    const int64_t N = (int64_t)p->n[0] * p->n[1] * p->n[2];
    const int64_t EN = N;                 // one image per bin
    const int64_t tot = (int64_t)p->B * EN;
    const int ncol = p->C;
    const int nb = 1024;
    DevBuf ksp, part, d2;
    TR_CUDA(cudaMalloc(&ksp.ptr, (size_t)std::max<int64_t>(p->total, 1) * ncol * sizeof(float2)));
    TR_CUDA(cudaMalloc(&part.ptr, 2 * nb * sizeof(double)));
    TR_CUDA(cudaMalloc(&d2.ptr, 2 * sizeof(double)));
    float2* kd = (float2*)ksp.ptr;
    double* pd = (double*)part.ptr;
    double* dd = (double*)d2.ptr;
    double h[2] = {0.0, 0.0};
    TR_TRY(norm2_async(x, tot, pd, nb, dd, st));
    TR_CUDA(cudaMemcpyAsync(h, dd, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    TR_CUDA(cudaStreamSynchronize(st));
    if (!(h[0] > 0.0) || !std::isfinite(h[0]))
        return fail(TR_ERR_INVALID_ARG, "tr_power_iteration: the start vector is zero or not finite");
    double lam = 0.0;
    for (int it = 0; it < n_iter; ++it) {
        k_scale<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(x, tot, dd);   // x <- x / ||x||
        TR_CHECK_LAUNCH();
        for (int b = 0; b < p->B; ++b)
            TR_TRY(nufft_forward_cols(p, b, x + b * EN, N, 1, p->maps, p->C, kInterpStore, 0.f, nullptr,
                                      kd + p->bins[b].offset * ncol, st));
        for (int b = 0; b < p->B; ++b)
            TR_TRY(nufft_adjoint_cols(p, b, kd + p->bins[b].offset * ncol, 1, p->maps, p->C, true, x + b * EN, N,
                                      st));
        TR_TRY(norm2_async(x, tot, pd, nb, dd, st));
        TR_CUDA(cudaMemcpyAsync(h, dd, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        TR_CUDA(cudaMemcpyAsync(p->err_host, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        TR_CUDA(cudaStreamSynchronize(st));
        if (*p->err_host != 0) {
            *p->err_host = 0;
            TR_CUDA(cudaMemsetAsync(p->dev_err, 0, sizeof(int), st));
            return fail(TR_ERR_TIMEOUT, "tr_power_iteration: a bounded device wait expired in step " +
                                            std::to_string(it));
        }
        if (!std::isfinite(h[0]))
            return fail(TR_ERR_NONFINITE, "tr_power_iteration: non-finite norm in step " + std::to_string(it));
        lam = std::sqrt(h[0]);  // ||A^H W A x|| with ||x|| = 1
    }
    // leave the normalised last iterate in x
    k_scale<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(x, tot, dd);
    TR_CHECK_LAUNCH();
    TR_CUDA(cudaStreamSynchronize(st));
    *norm_out = std::sqrt(lam);
    return TR_OK;
}

extern "C" tr_status tr_power_iteration(tr_plan* p, int32_t n_iter, void* work_images, double* norm_out,
                                        void* stream) {
    if (!p || !work_images || !norm_out || n_iter < 1)
        return fail(TR_ERR_INVALID_ARG, "tr_power_iteration: bad argument");
    if (!p->maps) return fail(TR_ERR_INVALID_ARG, "coil maps not set (tr_plan_set_maps)");
    DeviceGuard g(p->device);
    return power_impl(p, n_iter, (float2*)work_images, norm_out, (cudaStream_t)stream);
}
