// Batched line FFTs in shared memory (mixed radix 2/3/4/5/7/8, Stockham auto-sort).
//
// A CTA transforms W independent columns of length L held as smem[L][W]
// (column index fastest, so a warp touches whole 128-byte rows).  The stage
// indexing is the Stockham formulation of Govindaraju et al. (SC'08):
//   butterfly j < L/R reads   x[j + r L/R] * w_L^{(j mod Ns) r L/(Ns R)}
//                 writes  y[(j / Ns) Ns R + (j mod Ns) + r Ns] = DFT_R(...)[r]
// with Ns the product of the radices already applied.  The first stage reads
// through a caller functor (global memory with pad / shift / fused scaling) and
// the last stage writes through one (global memory with shift / crop, or a
// shared-memory epilogue), so an L-point FFT with S stages makes 2(S-1) passes
// over shared memory.  No normalisation is applied in either direction.
#pragma once

#include "tr_internal.cuh"

namespace tr {

// ------------------------------------------------------------------ async copies
// cp.async global -> shared; bytes < size zero-fills the rest (bytes may be 0).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int bytes) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
}

// ------------------------------------------------------------------ TMA tiles and mbarriers
// Tiled tensor copies (cp.async.bulk.tensor, no multicast) between global
// memory and a CTA's shared memory; loads complete on an mbarrier, stores are
// tracked with bulk groups.  Tensor maps are kernel parameters
// (__grid_constant__), built on the host per launch.
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
// First 128-byte boundary at or after p (TMA boxes start there; launches add 128 bytes of slack).
__device__ __forceinline__ float2* align128(unsigned char* p) {
    return reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(p) + 127) & ~uintptr_t(127));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity`; false after `limit` polls (each poll may
// suspend the thread for a hardware-defined time).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int limit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Bounded wait for phase `parity`; when it gives up, a second bounded wait
// (kMbarDrainLimit polls) lets the copies still in flight into this CTA's
// shared memory land before the caller abandons the tile, so no copy completes
// into shared memory the CTA no longer owns.  Returns the first wait's result.
__device__ __forceinline__ bool mbar_wait_or_drain(uint64_t* bar, unsigned parity, int limit) {
    if (mbar_wait_bounded(bar, parity, limit)) return true;
    mbar_wait_bounded(bar, parity, kMbarDrainLimit);
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];\n"
        ::"r"(smem_u32(dst)), "l"(tmap), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const void* tmap, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], [%2];\n"
        ::"r"(smem_u32(dst)), "l"(tmap), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void tma_store_3d(const void* tmap, const void* src, int x, int y, int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];\n"
                 ::"l"(tmap), "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void tma_store_4d(const void* tmap, const void* src, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];\n"
                 ::"l"(tmap), "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}
// contiguous global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// generic-proxy shared-memory writes -> visible to the TMA (async proxy)
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tma_store_commit_and_drain() {
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
__device__ __forceinline__ void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the issuing thread: every committed store group but the newest N has read its shared memory
template <int N>
__device__ __forceinline__ void tma_store_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}

// ------------------------------------------------------------------ thread-block clusters
// Distributed shared memory between the CTAs of a cluster (no TMA multicast).
__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size() {
    unsigned n;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
    return n;
}
// The address that `local` (this CTA's shared memory) has in CTA `rank` of the cluster.
__device__ __forceinline__ unsigned dsmem_addr(const void* local, unsigned rank) {
    unsigned remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_u32(local)), "r"(rank));
    return remote;
}
__device__ __forceinline__ float4 dsmem_load4(const void* local, unsigned rank) {
    float4 v;
    asm volatile("ld.shared::cluster.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(dsmem_addr(local, rank))
                 : "memory");
    return v;
}
__device__ __forceinline__ void dsmem_store4(void* local, unsigned rank, float4 v) {
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(dsmem_addr(local, rank)), "f"(v.x),
                 "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}
// Every thread of every CTA of the cluster: shared-memory stores (local or
// remote) before it are visible to loads after it.  A hardware barrier: the
// CTAs of a cluster are scheduled together.
__device__ __forceinline__ void cluster_sync_all() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// -i * z
__host__ __device__ __forceinline__ float2 mul_mi(float2 z) { return make_float2(z.y, -z.x); }
// +i * z
__host__ __device__ __forceinline__ float2 mul_pi(float2 z) { return make_float2(-z.y, z.x); }
// z * exp(-i theta) (forward) or z * exp(+i theta) (inverse), with c = cos theta, s = sin theta
__host__ __device__ __forceinline__ float2 crot(float2 z, float c, float s, bool inv) {
    return inv ? make_float2(fmaf(z.x, c, -z.y * s), fmaf(z.y, c, z.x * s))
               : make_float2(fmaf(z.x, c, z.y * s), fmaf(z.y, c, -z.x * s));
}

template <int R>
struct Dft;

template <>
struct Dft<2> {
    __host__ __device__ __forceinline__ static void run(float2 (&v)[2], bool) {
        float2 a = v[0], b = v[1];
        v[0] = cadd_p(a, b);
        v[1] = csub_p(a, b);
    }
};

template <>
struct Dft<4> {
    __host__ __device__ __forceinline__ static void run(float2 (&v)[4], bool inv) {
        float2 s0 = cadd_p(v[0], v[2]), d0 = csub_p(v[0], v[2]);
        float2 s1 = cadd_p(v[1], v[3]), d1 = csub_p(v[1], v[3]);
        float2 rd1 = inv ? mul_pi(d1) : mul_mi(d1);
        v[0] = cadd_p(s0, s1);
        v[2] = csub_p(s0, s1);
        v[1] = cadd_p(d0, rd1);
        v[3] = csub_p(d0, rd1);
    }
};

template <>
struct Dft<8> {
    __host__ __device__ __forceinline__ static void run(float2 (&v)[8], bool inv) {
        const float h = 0.70710678118654752f;
        float2 a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            a[r] = cadd_p(v[r], v[r + 4]);
            b[r] = csub_p(v[r], v[r + 4]);
        }
        // b_r *= w_8^r  (forward w_8 = (1 - i)/sqrt2)
        if (!inv) {
            b[1] = make_float2(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
            b[2] = mul_mi(b[2]);
            b[3] = make_float2(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
        } else {
            b[1] = make_float2(h * (b[1].x - b[1].y), h * (b[1].y + b[1].x));
            b[2] = mul_pi(b[2]);
            b[3] = make_float2(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y));
        }
        Dft<4>::run(a, inv);
        Dft<4>::run(b, inv);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
};

// Odd prime radices via conjugate-pair symmetry:
//   X_m     = v0 + sum_r cos(2 pi r m / R) s_r  -/+ i sum_r sin(2 pi r m / R) d_r
//   X_{R-m} = v0 + sum_r cos(2 pi r m / R) s_r  +/- i sum_r sin(2 pi r m / R) d_r
// with s_r = v_r + v_{R-r}, d_r = v_r - v_{R-r} (upper sign: forward).
template <int R>
struct OddTables;
template <>
struct OddTables<3> {
    __host__ __device__ __forceinline__ static float c(int k) { return -0.5f; }
    __host__ __device__ __forceinline__ static float s(int k) { return 0.86602540378443865f; }
};
template <>
struct OddTables<5> {
    __host__ __device__ __forceinline__ static float c(int k) {
        return k == 1 ? 0.30901699437494742f : -0.80901699437494742f;
    }
    __host__ __device__ __forceinline__ static float s(int k) {
        return k == 1 ? 0.95105651629515357f : 0.58778525229247313f;
    }
};
template <>
struct OddTables<7> {
    __host__ __device__ __forceinline__ static float c(int k) {
        return k == 1 ? 0.62348980185873353f : (k == 2 ? -0.22252093395631440f : -0.90096886790241913f);
    }
    __host__ __device__ __forceinline__ static float s(int k) {
        return k == 1 ? 0.78183148246802981f : (k == 2 ? 0.97492791218182361f : 0.43388373911755812f);
    }
};

template <int R>
struct DftOdd {
    __host__ __device__ __forceinline__ static void run(float2 (&v)[R], bool inv) {
        constexpr int H = (R - 1) / 2;
        float2 s[H + 1], d[H + 1];
#pragma unroll
        for (int r = 1; r <= H; ++r) {
            s[r] = cadd_p(v[r], v[R - r]);
            d[r] = csub_p(v[r], v[R - r]);
        }
        float2 out[R];
        float2 x0 = v[0];
#pragma unroll
        for (int r = 1; r <= H; ++r) x0 = cadd_p(x0, s[r]);
        out[0] = x0;
#pragma unroll
        for (int m = 1; m <= H; ++m) {
            float2 re = v[0], im = make_float2(0.f, 0.f);
#pragma unroll
            for (int r = 1; r <= H; ++r) {
                // angle index k = r*m mod R folded into [1, H] with a sign for the sine.
                int k = (r * m) % R;
                float sg = 1.f;
                if (k > H) { k = R - k; sg = -1.f; }
                float cv = OddTables<R>::c(k), sv = sg * OddTables<R>::s(k);
                re = cfma_real(cv, s[r], re);
                im = cfma_real(sv, d[r], im);
            }
            float2 t = inv ? mul_pi(im) : mul_mi(im);
            out[m] = cadd_p(re, t);
            out[R - m] = csub_p(re, t);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = out[r];
    }
};
template <>
struct Dft<3> : DftOdd<3> {};
template <>
struct Dft<5> : DftOdd<5> {};
template <>
struct Dft<7> : DftOdd<7> {};

// Composite radices for two-pass transforms (fewer shared-memory round trips).
// 16 = 4 x 4 (Cooley-Tukey): n = 4 n1 + n2, k = k1 + 4 k2,
//   X[k1 + 4 k2] = sum_n2 W16^(n2 k1) W4^(n2 k2) sum_n1 x[4 n1 + n2] W4^(n1 k1).
template <>
struct Dft<16> {
    __host__ __device__ __forceinline__ static void run(float2 (&v)[16], bool inv) {
        const float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f, h = 0.70710678118654752f;
        float2 a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            float2 t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            Dft<4>::run(t, inv);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
        }
        // twiddles W16^m, m = n2 k1 in {1, 2, 3, 4, 6, 9}
        a[1][1] = crot(a[1][1], c1, s1, inv);
        a[1][2] = crot(a[1][2], h, h, inv);
        a[1][3] = crot(a[1][3], s1, c1, inv);
        a[2][1] = crot(a[2][1], h, h, inv);
        a[2][2] = inv ? mul_pi(a[2][2]) : mul_mi(a[2][2]);
        a[2][3] = crot(a[2][3], -h, h, inv);
        a[3][1] = crot(a[3][1], s1, c1, inv);
        a[3][2] = crot(a[3][2], -h, h, inv);
        a[3][3] = crot(a[3][3], -c1, -s1, inv);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            Dft<4>::run(t, inv);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
        }
    }
};

// Coprime N1 x N2 (Good-Thomas prime-factor algorithm, no twiddles):
//   n = (N2 n1 + N1 n2) mod N,  k = (N2 t1 k1 + N1 t2 k2) mod N,
// t1 = N2^-1 mod N1, t2 = N1^-1 mod N2; then W_N^(n k) = W_N1^(n1 k1) W_N2^(n2 k2).
template <int N1, int N2, int T1, int T2>
struct DftPfa {
    __host__ __device__ __forceinline__ static void run(float2 (&v)[N1 * N2], bool inv) {
        constexpr int N = N1 * N2;
        float2 b[N2][N1];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) {
            float2 t[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) t[n1] = v[(N2 * n1 + N1 * n2) % N];
            Dft<N1>::run(t, inv);
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) b[n2][k1] = t[k1];
        }
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) {
            float2 t[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) t[n2] = b[n2][k1];
            Dft<N2>::run(t, inv);
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2) v[(N2 * T1 * k1 + N1 * T2 * k2) % N] = t[k2];
        }
    }
};
// 10 = 2 x 5: t1 = 5^-1 mod 2 = 1, t2 = 2^-1 mod 5 = 3
template <>
struct Dft<10> : DftPfa<2, 5, 1, 3> {};
// 20 = 4 x 5: t1 = 5^-1 mod 4 = 1, t2 = 4^-1 mod 5 = 4
template <>
struct Dft<20> : DftPfa<4, 5, 1, 4> {};

// One Stockham stage over every butterfly of every column.
template <int R, class Src, class Dst>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ tw, int L, int Ns, int W, bool inv,
                                          Src src, Dst dst) {
    const int nbf = L / R;
    const int step = L / (Ns * R);
    const int total = nbf * W;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int j = idx / W;
        const int w = idx - j * W;
        const int k = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 x = src(j + r * nbf, w);
            if (r > 0 && k > 0) {
                float2 t = tw[k * r * step];
                if (inv) t.y = -t.y;
                x = cmul_p(x, t);
            }
            v[r] = x;
        }
        Dft<R>::run(v, inv);
        const int d0 = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst(d0 + r * Ns, w, v[r]);
    }
}

template <class Src, class Dst>
__device__ __forceinline__ void fft_stage_dispatch(int R, const float2* tw, int L, int Ns, int W, bool inv,
                                                   Src src, Dst dst) {
    switch (R) {
        case 2: fft_stage<2>(tw, L, Ns, W, inv, src, dst); break;
        case 3: fft_stage<3>(tw, L, Ns, W, inv, src, dst); break;
        case 4: fft_stage<4>(tw, L, Ns, W, inv, src, dst); break;
        case 5: fft_stage<5>(tw, L, Ns, W, inv, src, dst); break;
        case 7: fft_stage<7>(tw, L, Ns, W, inv, src, dst); break;
        default: fft_stage<8>(tw, L, Ns, W, inv, src, dst); break;
    }
}

// ------------------------------------------------------------------ compile-time FFT
// Same Stockham stages, with L, W, the thread count and every radix, butterfly
// count, stride and twiddle step known at compile time (fully unrolled, no
// runtime division).  The radix sequence matches factor_radices() on the host:
// 7s, 5s, 3s first, then 8s, 4s, 2s.
__host__ __device__ constexpr int ct_radix(int L, int s) {
    int n = L, i = 0;
    for (int r : {7, 5, 3}) {
        while (n % r == 0) {
            if (i == s) return r;
            n /= r;
            ++i;
        }
    }
    for (int r : {8, 4, 2}) {
        while (n % r == 0) {
            if (i == s) return r;
            n /= r;
            ++i;
        }
    }
    return 0;
}
__host__ __device__ constexpr int ct_nstages(int L) {
    int s = 0;
    while (ct_radix(L, s) != 0) ++s;
    return s;
}
// Radix plans.  P = 0: the sequence above (L = 320 -> 5, 8, 8: three passes
// through shared memory).  P = 1: two passes where a composite radix exists
// (320 = 20 x 16, 160 = 10 x 16): each pass moves every element through
// shared memory once each way, and the transforms that are bound by the
// shared-memory data pipe lose a third of that traffic; other lengths keep P = 0.
__host__ __device__ constexpr int ct_radix_p(int P, int L, int s) {
    if (P == 1 && L == 320) return s == 0 ? 20 : (s == 1 ? 16 : 0);
    if (P == 1 && L == 160) return s == 0 ? 10 : (s == 1 ? 16 : 0);
    return ct_radix(L, s);
}
__host__ __device__ constexpr int ct_nstages_p(int P, int L) {
    int s = 0;
    while (ct_radix_p(P, L, s) != 0) ++s;
    return s;
}
// Row swizzle of a two-pass plan's intermediate tile.  With 64-byte rows (8
// columns) and an even first radix R0, the rows R0 j + r that the butterflies
// j and j + 1 of a half-warp write lie in the same half of the 32 banks (a
// 2-way conflict on every store); exchanging rows 2i and 2i + 1 within every
// odd block of R0 rows puts them in opposite halves, and the second pass reads
// its rows j + R0 r (four consecutive rows per warp) through the same map.
// Returns R0 where that applies, else 0 (no swizzle).
__host__ __device__ constexpr int ct_swz_p(int P, int L, int row_elems) {
    return (P == 1 && ct_nstages_p(P, L) == 2 && ct_radix_p(P, L, 0) % 2 == 0 && row_elems == 8)
               ? ct_radix_p(P, L, 0) : 0;
}
// (The map is m -> m ^ ((m / R0) & 1); at the stage 0 writes m / R0 is the
// butterfly index j, at the stage 1 reads it is the compile-time input index r.)

template <int L, int W, int NT, bool INV, int s, int Ns, bool LD = false, int P = 0>
struct CtStage {
    template <class Load, class Store>
    __device__ __forceinline__ static void run(const float2* __restrict__ src, float2* __restrict__ dst,
                                               const float2* __restrict__ tw, Load& load, Store& store) {
        constexpr int S = ct_nstages_p(P, L);
        constexpr int R = ct_radix_p(P, L, s);
        constexpr int NB = L / R;
        constexpr int TOTAL = NB * W;
        constexpr int STEP = L / (Ns * R);
        constexpr int ITERS = (TOTAL + NT - 1) / NT;
        constexpr int SW = ct_swz_p(P, L, W);          // stage 0 writes / stage 1 reads swizzled rows
#pragma unroll
        for (int it = 0; it < ITERS; ++it) {
            const int idx = (int)threadIdx.x + it * NT;
            if (TOTAL % NT == 0 || idx < TOTAL) {
                const int j = idx / W;
                const int w = idx - j * W;
                const int k = (Ns == 1) ? 0 : j % Ns;
                float2 v[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 x;
                    if constexpr (LD && s == 0) x = load(j + r * NB, w);
                    // stage 1: row j + NB r with j < NB = SW, so row / SW = r (a constant)
                    else x = src[((j + r * NB) ^ ((s == 1 && SW) ? (r & 1) : 0)) * W + w];
                    if (Ns > 1 && r > 0) {
                        float2 t = tw[k * r * STEP];
                        if (INV) t.y = -t.y;
                        x = cmul_p(x, t);
                    }
                    v[r] = x;
                }
                Dft<R>::run(v, INV);
                const int d0 = (Ns == 1) ? j * R : (j / Ns) * Ns * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (s == S - 1) store(d0 + r * Ns, w, v[r]);
                    // stage 0: row j SW + r with r < SW, so row / SW = j
                    else dst[((d0 + r * Ns) ^ ((s == 0 && SW) ? (j & 1) : 0)) * W + w] = v[r];
                }
            }
        }
        if constexpr (s < S - 1) {
            __syncthreads();
            CtStage<L, W, NT, INV, s + 1, Ns * R, LD, P>::run(dst, const_cast<float2*>(src), tw, load, store);
        }
    }
};

// Transform the [L][W] tile in A (A is clobbered); the last stage hands every
// output element to store(k, w, v).
struct NoLoad {
    __device__ __forceinline__ float2 operator()(int, int) const { return make_float2(0.f, 0.f); }
};
template <int L, int W, int NT, bool INV, class Store>
__device__ __forceinline__ void fft_ct(float2* A, float2* B, const float2* tw, Store& store) {
    NoLoad none;
    CtStage<L, W, NT, INV, 0, 1>::run(A, B, tw, none, store);
}
template <int P, int L, int W, int NT, bool INV, class Store>
__device__ __forceinline__ void fft_ct_p(float2* A, float2* B, const float2* tw, Store& store) {
    NoLoad none;
    CtStage<L, W, NT, INV, 0, 1, false, P>::run(A, B, tw, none, store);
}

// Same transform with the first stage reading its inputs from load(m, w)
// (input element m of column w) instead of A: A is not read, so it may hold
// whatever load() reads until the first stage ends.  The first stage writes B.
template <int L, int W, int NT, bool INV, class Load, class Store>
__device__ __forceinline__ void fft_ct_ld(float2* A, float2* B, const float2* tw, Load& load, Store& store) {
    CtStage<L, W, NT, INV, 0, 1, true>::run(A, B, tw, load, store);
}
template <int P, int L, int W, int NT, bool INV, class Load, class Store>
__device__ __forceinline__ void fft_ct_ld_p(float2* A, float2* B, const float2* tw, Load& load, Store& store) {
    CtStage<L, W, NT, INV, 0, 1, true, P>::run(A, B, tw, load, store);
}

// In-place variant: every stage first reads all of a thread's butterflies into
// registers, the CTA synchronises, and the results go back into the same
// [L][W] buffer; the last stage hands its outputs to store(k, w, v), which may
// write into the buffer.  Same butterflies, twiddles and output order as
// fft_ct (bit-identical results) with half the shared memory.
// RS: row stride of the buffer in elements (the W transformed columns are the
// first W of each row; RS > W transforms a column subset of a wider tile).
template <int L, int W, int NT, bool INV, int s, int Ns, int RS = W, int P = 0>
struct CtStageIP {
    template <class Store>
    __device__ __forceinline__ static void run(float2* buf, const float2* __restrict__ tw, Store& store) {
        constexpr int S = ct_nstages_p(P, L);
        constexpr int R = ct_radix_p(P, L, s);
        constexpr int NB = L / R;
        constexpr int TOTAL = NB * W;
        constexpr int STEP = L / (Ns * R);
        constexpr int ITERS = (TOTAL + NT - 1) / NT;
        constexpr int SW = ct_swz_p(P, L, RS);
        float2 v[ITERS][R];
#pragma unroll
        for (int it = 0; it < ITERS; ++it) {
            const int idx = (int)threadIdx.x + it * NT;
            if (TOTAL % NT == 0 || idx < TOTAL) {
                const int j = idx / W;
                const int w = idx - j * W;
                const int k = (Ns == 1) ? 0 : j % Ns;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 x = buf[((j + r * NB) ^ ((s == 1 && SW) ? (r & 1) : 0)) * RS + w];
                    if (Ns > 1 && r > 0) {
                        float2 t = tw[k * r * STEP];
                        if (INV) t.y = -t.y;
                        x = cmul_p(x, t);
                    }
                    v[it][r] = x;
                }
                Dft<R>::run(v[it], INV);
            }
        }
        __syncthreads();                                   // every read of this stage is done
#pragma unroll
        for (int it = 0; it < ITERS; ++it) {
            const int idx = (int)threadIdx.x + it * NT;
            if (TOTAL % NT == 0 || idx < TOTAL) {
                const int j = idx / W;
                const int w = idx - j * W;
                const int k = (Ns == 1) ? 0 : j % Ns;
                const int d0 = (Ns == 1) ? j * R : (j / Ns) * Ns * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (s == S - 1) store(d0 + r * Ns, w, v[it][r]);
                    else buf[((d0 + r * Ns) ^ ((s == 0 && SW) ? (j & 1) : 0)) * RS + w] = v[it][r];
                }
            }
        }
        if constexpr (s < S - 1) {
            __syncthreads();
            CtStageIP<L, W, NT, INV, s + 1, Ns * R, RS, P>::run(buf, tw, store);
        }
    }
};
template <int L, int W, int NT, bool INV, class Store>
__device__ __forceinline__ void fft_ct_ip(float2* buf, const float2* tw, Store& store) {
    CtStageIP<L, W, NT, INV, 0, 1>::run(buf, tw, store);
}
template <int P, int L, int W, int NT, bool INV, class Store>
__device__ __forceinline__ void fft_ct_ip_p(float2* buf, const float2* tw, Store& store) {
    CtStageIP<L, W, NT, INV, 0, 1, W, P>::run(buf, tw, store);
}
// The same on the first W columns of an [L][RS] buffer.
template <int L, int W, int RS, int NT, bool INV, class Store>
__device__ __forceinline__ void fft_ct_ip_rs(float2* buf, const float2* tw, Store& store) {
    CtStageIP<L, W, NT, INV, 0, 1, RS>::run(buf, tw, store);
}
template <int P, int L, int W, int RS, int NT, bool INV, class Store>
__device__ __forceinline__ void fft_ct_ip_rs_p(float2* buf, const float2* tw, Store& store) {
    CtStageIP<L, W, NT, INV, 0, 1, RS, P>::run(buf, tw, store);
}

// Buffer that the last stage of an L-point fft_ct does not read.
template <int L, int P = 0>
__device__ __forceinline__ float2* fft_ct_free(float2* A, float2* B) {
    return ((ct_nstages_p(P, L) - 1) % 2 == 0) ? B : A;
}

// Full transform: load(m, w) -> input element m of column w; store(k, w, v)
// receives output element k.  smA / smB are [L][W] scratch buffers.  The call
// ends with a __syncthreads() only between stages; callers that read smem
// written by `store` must synchronise themselves.
template <class Load, class Store>
__device__ __forceinline__ void fft_run(float2* smA, float2* smB, const float2* tw, const FftStages& S, int W,
                                        bool inv, Load load, Store store) {
    int Ns = 1;
    for (int s = 0; s < S.nstages; ++s) {
        const int R = S.radix[s];
        const bool first = (s == 0), last = (s == S.nstages - 1);
        float2* A = smA;
        float2* Bf = smB;
        auto smsrc = [A, W](int i, int w) { return A[i * W + w]; };
        auto smdst = [Bf, W](int i, int w, float2 v) { Bf[i * W + w] = v; };
        if (first && last) {
            fft_stage_dispatch(R, tw, S.L, Ns, W, inv, load, store);
        } else if (first) {
            fft_stage_dispatch(R, tw, S.L, Ns, W, inv, load, smdst);
        } else if (last) {
            fft_stage_dispatch(R, tw, S.L, Ns, W, inv, smsrc, store);
        } else {
            fft_stage_dispatch(R, tw, S.L, Ns, W, inv, smsrc, smdst);
        }
        if (!last) {
            __syncthreads();
            float2* t = smA;
            smA = smB;
            smB = t;
        }
        Ns *= R;
    }
}

}  // namespace tr
