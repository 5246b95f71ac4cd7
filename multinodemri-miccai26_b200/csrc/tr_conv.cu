// 3x3x3 convolutions (stride 1, zero padding 1) for the learned PDHG warm start:
// BF16 operands on the tensor cores (mma.sync m16n8k16), FP32 accumulation.
//
// Layout: activations channels-last (N, D, H, W, C) bf16; weights (Cout, 27, Cin)
// bf16 with tap t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1).
//   forward      y[v, co] = bias[co] + sum_{t, ci} w[co, t, ci] x[v + off_t, ci]
//                (the data gradient is the same kernel with w'[ci, 26 - t, co] = w[co, t, ci])
//   weight grad  dw[co, t, ci] = sum_v gy[v, co] x[v + off_t, ci]
//                split over voxel chunks into per-chunk partials, then a
//                fixed-order sum over chunks (deterministic).
// Implicit GEMM: forward M = voxels, N = Cout, K = 27 Cin; weight gradient
// M = Cin, N = Cout, K = voxels.  Requirements: Cin even, Cout % 8 == 0, Cout <= 128.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "tr_internal.cuh"

namespace {

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    const uint32_t l = *reinterpret_cast<const unsigned short*>(&lo);
    const uint32_t h = *reinterpret_cast<const unsigned short*>(&hi);
    return l | (h << 16);
}

struct ConvDims {
    int N, D, H, W, Cin, Cout;
    int64_t V;   // N*D*H*W
};

// Coordinates of a voxel, computed once per thread; neighbours then need only
// integer adds and bounds checks.
struct VoxelPos {
    int64_t v;
    int z, y, x;
};

__device__ __forceinline__ VoxelPos voxel_pos(const ConvDims& c, int64_t v) {
    VoxelPos p;
    p.v = v;
    int64_t r = v;
    p.x = (int)(r % c.W);
    r /= c.W;
    p.y = (int)(r % c.H);
    r /= c.H;
    p.z = (int)(r % c.D);
    return p;
}

__device__ __forceinline__ int64_t neighbour_at(const ConvDims& c, const VoxelPos& p, int dz, int dy, int dx) {
    const int zz = p.z + dz, yy = p.y + dy, xx = p.x + dx;
    if (zz < 0 || zz >= c.D || yy < 0 || yy >= c.H || xx < 0 || xx >= c.W) return -1;
    return p.v + ((int64_t)dz * c.H + dy) * c.W + dx;
}

// Forward: 4 warps, 64 voxels per CTA, each warp 16 voxels x Cout.
template <int NT>
__global__ void __launch_bounds__(128) k_conv3d_fwd(const __nv_bfloat16* __restrict__ x,
                                                    const __nv_bfloat16* __restrict__ w,
                                                    const float* __restrict__ bias, float* __restrict__ y,
                                                    ConvDims c) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int64_t m0 = ((int64_t)blockIdx.x * 4 + warp) * 16;
    const int64_t va = m0 + gid, vb = va + 8;
    float acc[NT][4];
#pragma unroll
    for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
    const int K27 = 27 * c.Cin;
    const VoxelPos pa = voxel_pos(c, va < c.V ? va : 0), pb = voxel_pos(c, vb < c.V ? vb : 0);
    for (int t = 0; t < 27; ++t) {
        const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
        const int64_t na = va < c.V ? neighbour_at(c, pa, dz, dy, dx) : -1;
        const int64_t nb = vb < c.V ? neighbour_at(c, pb, dz, dy, dx) : -1;
        const __nv_bfloat16* xa = x + (na < 0 ? 0 : na * c.Cin);
        const __nv_bfloat16* xb = x + (nb < 0 ? 0 : nb * c.Cin);
        for (int ci0 = 0; ci0 < c.Cin; ci0 += 16) {
            const int k0 = ci0 + tig * 2, k1 = k0 + 8;
            const bool v0 = k0 < c.Cin, v1 = k1 < c.Cin;
            const uint32_t a0 = (na >= 0 && v0) ? ld_pair(xa + k0) : 0u;
            const uint32_t a1 = (nb >= 0 && v0) ? ld_pair(xb + k0) : 0u;
            const uint32_t a2 = (na >= 0 && v1) ? ld_pair(xa + k1) : 0u;
            const uint32_t a3 = (nb >= 0 && v1) ? ld_pair(xb + k1) : 0u;
#pragma unroll
            for (int n = 0; n < NT; ++n) {
                const __nv_bfloat16* wr = w + (int64_t)(n * 8 + gid) * K27 + t * c.Cin;
                const uint32_t b0 = v0 ? ld_pair(wr + k0) : 0u;
                const uint32_t b1 = v1 ? ld_pair(wr + k1) : 0u;
                mma_bf16(acc[n], a0, a1, a2, a3, b0, b1);
            }
        }
    }
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const int co = n * 8 + tig * 2;
        const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
        if (va < c.V) {
            y[va * c.Cout + co] = acc[n][0] + b0;
            y[va * c.Cout + co + 1] = acc[n][1] + b1;
        }
        if (vb < c.V) {
            y[vb * c.Cout + co] = acc[n][2] + b0;
            y[vb * c.Cout + co + 1] = acc[n][3] + b1;
        }
    }
}

constexpr int kWgradChunk = 2048;   // voxels per CTA

// Weight gradient partials: grid (chunks, 27 taps, ceil(Cin / 64)); warp w owns
// input channels [64 z + 16 w, +16) and all Cout outputs.
template <int NT>
__global__ void __launch_bounds__(128) k_conv3d_wgrad(const __nv_bfloat16* __restrict__ x,
                                                      const __nv_bfloat16* __restrict__ gy,
                                                      float* __restrict__ part, ConvDims c) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int t = blockIdx.y;
    const int ci0 = blockIdx.z * 64 + warp * 16;
    if (ci0 >= c.Cin) return;
    const int64_t vbeg = (int64_t)blockIdx.x * kWgradChunk;
    const int64_t vend = min(vbeg + kWgradChunk, c.V);
    const int ra = ci0 + gid, rb = ra + 8;
    const bool oka = ra < c.Cin, okb = rb < c.Cin;
    float acc[NT][4];
#pragma unroll
    for (int n = 0; n < NT; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
    // this thread's four voxels k = 2tig, 2tig+1, 2tig+8, 2tig+9 of each 16-voxel step,
    // with coordinates advanced incrementally (16 voxels per step along x, then y, z, volume)
    VoxelPos pos[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) pos[j] = voxel_pos(c, min(vbeg + tig * 2 + (j & 1) + (j >> 1) * 8, c.V - 1));
    for (int64_t kb = vbeg; kb < vend; kb += 16) {
        int64_t nbr[4];
        bool in[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t v = kb + tig * 2 + (j & 1) + (j >> 1) * 8;
            in[j] = v < vend;
            nbr[j] = in[j] ? neighbour_at(c, pos[j], dz, dy, dx) : -1;
            // advance to v + 16
            pos[j].v += 16;
            pos[j].x += 16;
            while (pos[j].x >= c.W) {
                pos[j].x -= c.W;
                if (++pos[j].y >= c.H) {
                    pos[j].y = 0;
                    if (++pos[j].z >= c.D) pos[j].z = 0;      // next volume of the batch
                }
            }
        }
        __nv_bfloat16 xa[4], xb[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            xa[j] = (nbr[j] >= 0 && oka) ? x[nbr[j] * c.Cin + ra] : zero;
            xb[j] = (nbr[j] >= 0 && okb) ? x[nbr[j] * c.Cin + rb] : zero;
        }
        const uint32_t a0 = pack_bf16(xa[0], xa[1]), a1 = pack_bf16(xb[0], xb[1]);
        const uint32_t a2 = pack_bf16(xa[2], xa[3]), a3 = pack_bf16(xb[2], xb[3]);
#pragma unroll
        for (int n = 0; n < NT; ++n) {
            const int co = n * 8 + gid;
            __nv_bfloat16 g[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int64_t v = kb + tig * 2 + (j & 1) + (j >> 1) * 8;
                g[j] = in[j] ? gy[v * c.Cout + co] : zero;
            }
            mma_bf16(acc[n], a0, a1, a2, a3, pack_bf16(g[0], g[1]), pack_bf16(g[2], g[3]));
        }
    }
    // part[chunk][t][ci][co]
    float* dst = part + (((int64_t)blockIdx.x * 27 + t) * c.Cin) * c.Cout;
#pragma unroll
    for (int n = 0; n < NT; ++n) {
        const int co = n * 8 + tig * 2;
        if (oka) {
            dst[(int64_t)ra * c.Cout + co] = acc[n][0];
            dst[(int64_t)ra * c.Cout + co + 1] = acc[n][1];
        }
        if (okb) {
            dst[(int64_t)rb * c.Cout + co] = acc[n][2];
            dst[(int64_t)rb * c.Cout + co + 1] = acc[n][3];
        }
    }
}

// dw[co][t][ci] = sum over chunks (in order) of part[chunk][t][ci][co]
__global__ void k_wgrad_reduce(const float* __restrict__ part, float* __restrict__ dw, int nchunks, int Cin,
                               int Cout) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)Cout * 27 * Cin;
    if (i >= total) return;
    const int ci = (int)(i % Cin);
    const int t = (int)((i / Cin) % 27);
    const int co = (int)(i / (27LL * Cin));
    const int64_t stride = 27LL * Cin * Cout;
    const int64_t off = ((int64_t)t * Cin + ci) * Cout + co;
    float s = 0.f;
    for (int k = 0; k < nchunks; ++k) s += part[k * stride + off];
    dw[i] = s;
}

tr_status check_dims(const ConvDims& c) {
    if (c.N < 1 || c.D < 1 || c.H < 1 || c.W < 1) return tr::fail(TR_ERR_INVALID_ARG, "conv3d: empty volume");
    if (c.Cin < 2 || (c.Cin & 1)) return tr::fail(TR_ERR_INVALID_ARG, "conv3d: Cin must be even and >= 2");
    if (c.Cout < 8 || (c.Cout % 8) || c.Cout > 128)
        return tr::fail(TR_ERR_INVALID_ARG, "conv3d: Cout must be a multiple of 8 in [8, 128]");
    return TR_OK;
}

}  // namespace

extern "C" tr_status tr_conv3d_fwd(const void* x, const void* w, const float* bias, float* y, int32_t N, int32_t D,
                                   int32_t H, int32_t W, int32_t Cin, int32_t Cout, void* stream) {
    if (!x || !w || !y) return tr::fail(TR_ERR_INVALID_ARG, "tr_conv3d_fwd: null pointer");
    ConvDims c{N, D, H, W, Cin, Cout, (int64_t)N * D * H * W};
    TR_TRY(check_dims(c));
    const unsigned blocks = (unsigned)((c.V + 63) / 64);
    cudaStream_t st = (cudaStream_t)stream;
    const auto* xb = (const __nv_bfloat16*)x;
    const auto* wb = (const __nv_bfloat16*)w;
    switch (Cout / 8) {
#define TR_CONV_CASE(NTV) \
    case NTV: k_conv3d_fwd<NTV><<<blocks, 128, 0, st>>>(xb, wb, bias, y, c); break;
        TR_CONV_CASE(1) TR_CONV_CASE(2) TR_CONV_CASE(3) TR_CONV_CASE(4) TR_CONV_CASE(5) TR_CONV_CASE(6)
        TR_CONV_CASE(7) TR_CONV_CASE(8) TR_CONV_CASE(9) TR_CONV_CASE(10) TR_CONV_CASE(11) TR_CONV_CASE(12)
        TR_CONV_CASE(13) TR_CONV_CASE(14) TR_CONV_CASE(15) TR_CONV_CASE(16)
#undef TR_CONV_CASE
        default: return tr::fail(TR_ERR_INVALID_ARG, "conv3d: bad Cout");
    }
    TR_CHECK_LAUNCH();
    return TR_OK;
}

extern "C" tr_status tr_conv3d_wgrad_workspace(int32_t N, int32_t D, int32_t H, int32_t W, int32_t Cin,
                                               int32_t Cout, size_t* bytes) {
    if (!bytes) return tr::fail(TR_ERR_INVALID_ARG, "null bytes");
    const int64_t V = (int64_t)N * D * H * W;
    const int64_t chunks = (V + kWgradChunk - 1) / kWgradChunk;
    *bytes = (size_t)(chunks * 27 * (int64_t)Cin * Cout * sizeof(float));
    return TR_OK;
}

extern "C" tr_status tr_conv3d_wgrad(const void* x, const void* gy, float* dw, int32_t N, int32_t D, int32_t H,
                                     int32_t W, int32_t Cin, int32_t Cout, void* workspace, size_t workspace_bytes,
                                     void* stream) {
    if (!x || !gy || !dw || !workspace) return tr::fail(TR_ERR_INVALID_ARG, "tr_conv3d_wgrad: null pointer");
    ConvDims c{N, D, H, W, Cin, Cout, (int64_t)N * D * H * W};
    TR_TRY(check_dims(c));
    size_t need = 0;
    tr_conv3d_wgrad_workspace(N, D, H, W, Cin, Cout, &need);
    if (workspace_bytes < need) return tr::fail(TR_ERR_INVALID_ARG, "tr_conv3d_wgrad: workspace too small");
    const int64_t chunks = (c.V + kWgradChunk - 1) / kWgradChunk;
    cudaStream_t st = (cudaStream_t)stream;
    dim3 grid((unsigned)chunks, 27, (unsigned)((Cin + 63) / 64));
    const auto* xb = (const __nv_bfloat16*)x;
    const auto* gb = (const __nv_bfloat16*)gy;
    float* part = (float*)workspace;
    switch (Cout / 8) {
#define TR_WG_CASE(NTV) \
    case NTV: k_conv3d_wgrad<NTV><<<grid, 128, 0, st>>>(xb, gb, part, c); break;
        TR_WG_CASE(1) TR_WG_CASE(2) TR_WG_CASE(3) TR_WG_CASE(4) TR_WG_CASE(5) TR_WG_CASE(6) TR_WG_CASE(7)
        TR_WG_CASE(8) TR_WG_CASE(9) TR_WG_CASE(10) TR_WG_CASE(11) TR_WG_CASE(12) TR_WG_CASE(13) TR_WG_CASE(14)
        TR_WG_CASE(15) TR_WG_CASE(16)
#undef TR_WG_CASE
        default: return tr::fail(TR_ERR_INVALID_ARG, "conv3d: bad Cout");
    }
    TR_CHECK_LAUNCH();
    const int64_t total = (int64_t)Cout * 27 * Cin;
    k_wgrad_reduce<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(part, dw, (int)chunks, Cin, Cout);
    TR_CHECK_LAUNCH();
    return TR_OK;
}
