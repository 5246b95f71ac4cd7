/*
 * toporecon_b200 -- C ABI of the Blackwell (sm_100a) backend for toporecon's
 * PDHG reconstruction loop (TVM / TVME / TVMW).
 *
 * Reference interfaces replaced (paths inside MRI-Research/MultiNodeMRI-MICCAI26):
 *   NufftBackend contract ............ src/toporecon/nufft_backend.py:11-52
 *   SigPyNufftBackend.__init__ ....... src/toporecon/nufft_backend.py:58-88
 *   SigPyNufftBackend.forward ........ src/toporecon/nufft_backend.py:101-107
 *   SigPyNufftBackend.adjoint ........ src/toporecon/nufft_backend.py:109-116
 *   data dual step (b,c,e loop) ...... src/toporecon/algorithms/tvme.py:256-267
 *   coil-combined adjoint ............ src/toporecon/algorithms/tvme.py:382-394
 *   TvmReconstructor.pdhg ............ src/toporecon/algorithms/tvm.py:227-380
 *   TvmeReconstructor.pdhg ........... src/toporecon/algorithms/tvme.py:208-482
 *   TvmwReconstructor.pdhg ........... src/toporecon/algorithms/tvmw.py:385-685
 *   *Reconstructor.run tolerance ..... src/toporecon/algorithms/tvme.py:512-557,
 *                                      tvm.py:406-472, tvmw.py:716-773
 *
 * Conventions
 *   - Complex data are interleaved float pairs (numpy complex64 / torch.cfloat).
 *   - Images are C-order (..., Z, Y, X); coordinates are (M, 3) ordered z, y, x
 *     in grid units (the reference's internal convention, nufft_backend.py:14-16).
 *   - Every entry point returns a tr_status; none aborts or throws.  The text of
 *     the last failure on the calling thread is returned by tr_last_error_string.
 *   - Device pointers belong to the caller.  A plan owns only its sorted copy of
 *     the trajectory, its permutation and tile tables, its coil maps and its
 *     FFT/gridding workspace, all freed by tr_plan_destroy.
 *   - All work is enqueued on the caller's stream (cudaStream_t passed as void*);
 *     a plan is used by one stream at a time.
 */
#ifndef TOPORECON_B200_H
#define TOPORECON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t tr_status;
#define TR_OK 0
#define TR_ERR_INVALID_ARG 1  /* bad shape, pointer, bin index (reference: ValueError / IndexError) */
#define TR_ERR_OOM 2          /* device allocation failed */
#define TR_ERR_NONFINITE 3    /* a tolerance reduction saw NaN/Inf */
#define TR_ERR_TIMEOUT 4      /* a bounded device-side wait expired */
#define TR_ERR_CUDA 5         /* any other CUDA runtime failure */
#define TR_ERR_UNSUPPORTED 6  /* legal but unsupported configuration */

#define TR_ALG_TVM 0
#define TR_ALG_TVME 1
#define TR_ALG_TVMW 2

typedef struct tr_plan tr_plan;

/* Plan description (replaces SigPyNufftBackend(img_shape, coordinates, device),
 * nufft_backend.py:58-88, for every local motion bin at once). */
typedef struct {
    int32_t img_shape[3];        /* Z, Y, X; each >= 10 */
    int32_t n_bins;              /* >= 1 */
    const int64_t* bin_counts;   /* host [n_bins]: samples per bin (TR_b * RO) */
    const float* coords;         /* host [sum(bin_counts) * 3]: zyx grid units, bins concatenated */
    const float* dcf;            /* host [sum(bin_counts)] density weights, or NULL (all ones) */
    int32_t n_coils;             /* C >= 1 (columns per echo on the batched path) */
    int32_t n_echoes;            /* E >= 1 */
    float oversamp;              /* must be 1.25 (SigPy default used by the reference) */
    int32_t width;               /* must be 4 (SigPy default used by the reference) */
    int32_t device;              /* CUDA device ordinal */
    int32_t flags;               /* TR_PLAN_* bits */
} tr_plan_desc;

#define TR_PLAN_AUTOTUNE 1       /* time candidate launch shapes at plan creation */
#define TR_PLAN_NO_TMA 2         /* stage FFT tiles with cp.async instead of TMA (comparison runs) */
#define TR_PLAN_YZ_FUSION 4      /* run the y and z FFT passes as one cluster kernel where the geometry
                                    allows (comparison runs: measured slower than the separate passes) */
#define TR_PLAN_THREE_PASS_320 8 /* run the 320-point FFT passes (x and the line passes) in three
                                    shared-memory passes (radices 5, 8, 8) instead of two (20, 16)
                                    (comparison runs; results agree to float rounding) */
#define TR_PLAN_NO_COLUMN_SKIP 16 /* transform every z line of the grid, also those of (y, x) tile columns
                                    that no sample's kernel reaches (comparison runs; same results) */

typedef struct {
    int32_t os_shape[3];         /* oversampled grid (ceil(1.25 n) per axis) */
    int64_t total_samples;
    int64_t workspace_bytes;     /* device bytes owned by the plan */
    int32_t wavelet_levels;      /* db6 levels for TVMW (PyWavelets max level) */
    int64_t wavelet_coeffs;      /* db6 coefficients per (bin, echo) image */
    int32_t fft_line_width;      /* columns per CTA chosen for the FFT passes */
    int32_t spread_columns;      /* k-space columns per gridding CTA (last tuned / used value) */
} tr_plan_info_t;

tr_status tr_plan_create(const tr_plan_desc* desc, tr_plan** out);
tr_status tr_plan_destroy(tr_plan* plan);
tr_status tr_plan_info(const tr_plan* plan, tr_plan_info_t* info);
const char* tr_last_error_string(void);

/* Bounded device waits.  Kernels that stage tiles by TMA wait for them on an
 * mbarrier for at most `polls` polls (default 1 << 20); a wait that gives up
 * lets the copies already in flight land, marks the plan's device error word
 * and leaves its tile, and the next tr_pdhg_run / tr_pdhg_phase returns
 * TR_ERR_TIMEOUT with the results of that iteration invalid.  polls = 0 makes
 * every such wait give up at once, which exercises that error path without a
 * fault.  Drops the plan's captured iteration graph.  (No counterpart in the
 * reference, whose CuPy kernels have no device-side waits.) */
tr_status tr_plan_set_wait_limit(tr_plan* plan, int32_t polls);

/* Coil sensitivities (C, Z, Y, X) complex64 on the device; copied into the
 * plan's coil-interleaved layout.  Needed by the batched path only. */
tr_status tr_plan_set_maps(tr_plan* plan, const void* mps, void* stream);

/* Sample order conversion for one bin.
 * External: (ncol, M_b) acquisition order (the reference's per-bin (E, C, TR_b, RO)).
 * Internal: (M_b, ncol) tile-sorted, columns interleaved. */
tr_status tr_plan_sort_kspace(tr_plan* plan, int32_t bin, const void* ext, void* internal,
                              int32_t ncol, void* stream);
tr_status tr_plan_unsort_kspace(tr_plan* plan, int32_t bin, const void* internal, void* ext,
                                int32_t ncol, void* stream);

/* Drop-in single-image NUFFT: NufftBackend.forward(image, bin) / .adjoint(ksp, bin)
 * (nufft_backend.py:101-116).  image (Z, Y, X), ksp (M_b) in acquisition order.
 * The adjoint applies no density weights (the caller passes dcf*q as the
 * reference does, tvme.py:389-391). */
tr_status tr_nufft_forward(tr_plan* plan, int32_t bin, const void* image, void* ksp, void* stream);
tr_status tr_nufft_adjoint(tr_plan* plan, int32_t bin, const void* ksp, void* image, void* stream);

/* Batched coil/echo NUFFT on the internal layout (the PDHG hot path).
 * forward: ksp[m, e, c] = F_b(images[e] * S_c)[m]            (images (E, Z, Y, X))
 * adjoint: images[e] = sum_c conj(S_c) F_b^H(w[m] * ksp[m, e, c]),
 *          w = plan dcf when use_dcf != 0, else 1. */
tr_status tr_nufft_forward_bin(tr_plan* plan, int32_t bin, const void* images, void* ksp_internal,
                               void* stream);
tr_status tr_nufft_adjoint_bin(tr_plan* plan, int32_t bin, const void* ksp_internal, int32_t use_dcf,
                               void* images, void* stream);

/* PDHG (one device; all motion bins and echoes resident). */
typedef struct {
    int32_t algorithm;           /* TR_ALG_* */
    int32_t l2_coupling;         /* --l2-coupling: prox over all echoes of the motion dual */
    float sigma, tau;            /* dual / primal steps (reference: 1/6, tvme.py:968); sigma is the
                                    step of the TV and wavelet duals */
    float lam_m;                 /* motion TV (TVM lamda, TVME lamda_m, TVMW lambda1) */
    float lam_e;                 /* TVME echo-spatial TV (lamda_e) */
    float lam_w1;                /* TVMW db1 echo wavelet (lambda2) */
    float lam_w2;                /* TVMW db6 spatial wavelet (lambda3) */
    int32_t use_graph;           /* capture one iteration in a CUDA graph and replay it */
    float sigma_data;            /* step of the data dual q; 0 means sigma (the reference's single
                                    step, tvme.py:263-267).  A separate value gives block-diagonal
                                    PDHG steps (no counterpart in the reference). */
} tr_pdhg_params;

/* Device state, all (B, E, Z, Y, X) complex64 unless noted; unused fields NULL.
 *   TVM / TVME: u = u_now, u_bar = the extrapolated iterate (the returned image).
 *   TVMW:       u = primal_u_tmp, u_bar = primal_u (extrapolated, returned).
 * q and y use the internal k-space layout, bins concatenated (bin offsets as in
 * tr_plan_bin_offset * E * C).  g is scratch for the coil-combined adjoint;
 * w2adj is TVMW scratch; p_w2 is (B*E, wavelet_coeffs). */
typedef struct {
    void* u;
    void* u_bar;
    void* p_m;
    void* p_ex;
    void* p_ey;
    void* p_ez;
    void* p_w1;
    void* p_w2;
    void* w2adj;
    void* q;
    const void* y;
    void* g;
} tr_pdhg_state;

tr_status tr_plan_bin_offset(const tr_plan* plan, int32_t bin, int64_t* offset, int64_t* count);

/* Runs up to max_iters iterations; stops after the first iteration whose
 * tolerance is below tol (tvme.py:555, tvm.py:466, tvmw.py:772).
 * tol_history (host, >= max_iters doubles, may be NULL) receives each
 * iteration's tolerance; iters_done the number of iterations run. */
tr_status tr_pdhg_run(tr_plan* plan, const tr_pdhg_state* state, const tr_pdhg_params* params,
                      int32_t max_iters, double tol, double* tol_history, int32_t* iters_done,
                      void* stream);

/* Bin-sharded PDHG: the motion bins of one problem spread over ranks, each
 * rank with a plan holding a contiguous range of bins.  Replaces the
 * reference's motion-axis halo exchange (u_bar forward ghost around the motion
 * dual, tvme.py:217-229, tvm.py:230-260; p_m backward ghost around the motion
 * divergence, tvme.py:421-437, tvm.py:342-357, tvmw.py:662-670) and the
 * all-reduce of the stopping sums (tvme.py:518-551, tvm.py:406-472,
 * tvmw.py:716-769). */
typedef struct {
    int32_t n_bins_global;       /* bins of the whole problem (>= bin_offset + the plan's bins) */
    int32_t bin_offset;          /* global index of the plan's first bin */
    const void* u_bar_next;      /* device (E, Z, Y, X) complex64: u_bar of the global bin after the plan's
                                    last one; NULL when the plan holds the global last bin */
    const void* p_m_prev;        /* device (E, Z, Y, X) complex64: p_m of the global bin before the plan's
                                    first one; NULL when the plan holds bin 0 */
} tr_pdhg_shard;

/* One half of a PDHG iteration on the plan's bins, asynchronous on `stream`.
 * phase 1: every dual update (data, motion / echo TV, wavelets) and the data
 *          gradient; reads shard->u_bar_next.
 * phase 2: primal update, extrapolation and the FP64 tolerance sums
 *          (numerator, denominator) of the plan's bins into tol_sums[2]
 *          (device memory) for the caller's all-reduce; reads shard->p_m_prev.
 * phase 3: the part of phase 1 that reads only this plan's state (TVMW
 *          spatial-wavelet dual, data dual with its forward NUFFTs);
 * phase 4: the rest of phase 1 (TV / W1 duals, data gradient); reads
 *          shard->u_bar_next.  Phases 3 then 4 do exactly what phase 1 does,
 *          so a caller can enqueue 3 while the u_bar halo is in flight.
 * Between the phases the caller passes its last p_m bin to the next rank; after
 * phase 2 its first u_bar bin to the previous rank.  TR_ERR_TIMEOUT reports a
 * device wait that expired in an earlier phase on this plan. */
tr_status tr_pdhg_phase(tr_plan* plan, const tr_pdhg_state* state, const tr_pdhg_params* params,
                        const tr_pdhg_shard* shard, int32_t phase, double* tol_sums, void* stream);

/* Operator norm of the data term for the PDHG step rule: sqrt(||A^H W A||)
 * (A = [F_b S_c] over every bin, echo and coil; W = density weights) by
 * n_iter power-iteration steps.  The operator is block diagonal over (bin,
 * echo) with the same block for every echo of a bin, so the iterate is one
 * image per bin: caller scratch work_images (B, Z, Y, X), which must hold a
 * nonzero start and holds the last normalised iterate on return.  Norms are
 * reduced in FP64; the k-space scratch (total samples x C complex64) is
 * allocated and freed inside.
 * No counterpart in the reference (it fixes sigma = tau = 1/6, tvme.py:968). */
tr_status tr_power_iteration(tr_plan* plan, int32_t n_iter, void* work_images, double* norm_out,
                             void* stream);

/* TVMW spatial wavelet W2 of every (bin, echo) image of the plan: db6, zero
 * mode, PyWavelets' maximum level (tr_plan_info: wavelet_levels / _coeffs).
 *   forward: coeffs (B*E, wavelet_coeffs) = wavedec3(images (B, E, Z, Y, X)),
 *            per image [cA_L | 7 detail bands of level L | ... | level 1],
 *            bands aad, ada, add, daa, dad, dda, ddd (letters z, y, x)
 *   adjoint: images = waverec3(coeffs) cropped to (Z, Y, X), the operator the
 *            reference applies in place of the adjoint.
 * Replaces PtwtWaveletOps.w2_fwd / w2_adj (tvmw.py:196-206). */
tr_status tr_wavelet_forward(tr_plan* plan, const void* images, void* coeffs, void* stream);
tr_status tr_wavelet_adjoint(tr_plan* plan, const void* coeffs, void* images, void* stream);

/* Per-stage device time of the batched NUFFT of one bin (all E x C columns):
 * ms[10] and the algorithmic bytes[10] of each stage, in the order
 * forward x, y, z, interpolation(+dual prox), gridding, adjoint z, y, x,
 * fused forward y + z, fused adjoint z + y.  The last two are 0 ms / 0 bytes
 * when the plan runs the separate passes; when it fuses them, the separate y
 * and z passes are still timed for comparison.
 * Each stage is run reps times after one warm-up; used for roofline reports.
 * Replaces the reference's wall-clock timers (tvme.py:509, :561-567). */
tr_status tr_profile_nufft(tr_plan* plan, int32_t bin, int32_t reps, double* ms, double* bytes, void* stream);

/* 3x3x3 convolutions of the learned PDHG warm start (no counterpart in the
 * reference, which always starts PDHG from zeros: tvme.py:190-205).  BF16
 * tensor-core operands, FP32 accumulation; stride 1, zero padding 1.
 * Activations channels-last (N, D, H, W, C) bf16, weights (Cout, 27, Cin)
 * bf16 (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)); Cin even, Cout % 8 == 0, <= 128.
 *   forward:     y (N, D, H, W, Cout) f32 = conv(x, w) + bias (bias may be NULL)
 *   weight grad: dw (Cout, 27, Cin) f32 = sum_v gy[v, co] x[v + tap, ci]
 *                (deterministic; needs tr_conv3d_wgrad_workspace bytes of scratch)
 * The data gradient is tr_conv3d_fwd with the flipped, channel-swapped weights. */
tr_status tr_conv3d_fwd(const void* x, const void* w, const float* bias, float* y, int32_t N, int32_t D,
                        int32_t H, int32_t W, int32_t Cin, int32_t Cout, void* stream);
tr_status tr_conv3d_wgrad_workspace(int32_t N, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                                    size_t* bytes);
tr_status tr_conv3d_wgrad(const void* x, const void* gy, float* dw, int32_t N, int32_t D, int32_t H, int32_t W,
                          int32_t Cin, int32_t Cout, void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free stopping-tolerance sums (no counterpart in the reference).
 * For callers that cannot allocate device memory where they run the stopping
 * test -- hosts that own the whole device heap through their own allocator and
 * forbid cudaMalloc from a library -- this computes in FP64 what tr_pdhg_run's
 * tolerance step computes, without a plan and without allocating:
 *   TVM / TVME: sums_out = { sum |cur - prev|^2, sum |cur|^2 }
 *   TVMW:       sums_out = { sum |prev - cur|^2, sum |prev|^2 }
 * (tolerance = sqrt(s0) / sqrt(s1), resp. / max(sqrt(s1), 1e-12)).
 * cur, prev: n complex64 values on the current device; sums_out: 2 doubles
 * on the device, written asynchronously on `stream`.
 * Limit: n <= TR_NOALLOC_MAX_ELEMS (larger n returns TR_ERR_INVALID_ARG).
 * The partial sums live in a 64 KiB file-scope device array that every GPU
 * loading the library keeps until exit; calls share it, so calls whose
 * kernels may overlap on the GPU race and must be ordered by the caller.
 * The first call on a device looks up that array's device address (a
 * runtime call, no allocation); make that first call before any stream
 * capture on the device. */
#define TR_NOALLOC_MAX_ELEMS (64LL * 1024 * 1024)
tr_status tr_tolerance_sums_noalloc(const void* cur, const void* prev, int64_t n, int32_t algorithm,
                                    double* sums_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TOPORECON_B200_H */
