"""GPU parity of the batched NUFFT at the benchmark's own geometry.

The TVME benchmark workload is a 128 x 256 x 256 image (160 x 320 x 320 grid)
with 6 echoes x 16 coils = 96 k-space columns per sample.  At that size the
forward and adjoint run kernels no smaller test reaches: the y passes at
L = 320 with 8 columns per CTA, the z passes at L = 160 with 16, the TMA x
passes over twelve 8-coil groups, and gridding over 96 columns with the
k-space centre's tiles split into list ranges.  The GPU computes all 96
columns; the CPU oracle (SigPy 0.1.27 restatement, C/OpenMP loops) checks
three whole echoes (48 columns, first, middle and last column groups) at the
1e-4 relative-L2 bar of the reference NUFFT (nufft_backend.py:101-116).
"""

import numpy as np
import pytest

from _fixtures import pkg
from oracle import cgrid
from oracle import nufft as onf

pytestmark = pytest.mark.gpu

TOL_NUFFT = 1e-4
SHAPE = (128, 256, 256)
E, C = 6, 16
CHECK_ECHOES = (0, 3, 5)


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def problem():
    torch = _torch()
    syn = pkg("synthetic")
    nb = pkg("nufft_backend")
    rng = np.random.default_rng(2026)
    # 64 whole cones of the benchmark trajectory (51,200 samples): every cone
    # starts at the k-space centre, so the centre tiles exceed one list range
    k = syn.cones_trajectory(SHAPE, 4096, 800, rng)[:64].reshape(-1, 3)
    edge = np.array([[0.0, 0.0, 0.0], [-64.0, -128.0, -128.0], [63.999, 0.5, -0.25], [1.0, -2.0, 3.0]],
                    dtype=np.float32)
    k = np.concatenate([edge, k]).astype(np.float32)
    dcf = syn.density(k, SHAPE)
    mps = syn.coil_maps(SHAPE, C, rng)
    img = (rng.standard_normal((E,) + SHAPE, dtype=np.float32)
           + 1j * rng.standard_normal((E,) + SHAPE, dtype=np.float32)).astype(np.complex64)
    be = nb.B200NufftBackend(SHAPE, [k], 0, dcf=[dcf], n_coils=C, n_echoes=E, autotune=True)
    be.set_maps(mps)
    assert be.os_shape == (160, 320, 320)
    yield torch, be, k, dcf, mps, img, rng
    be.close()


def test_forward_96_columns_matches_oracle(problem):
    torch, be, k, dcf, mps, img, rng = problem
    ks = be.forward_bin(torch.from_numpy(img).cuda(), 0)                # (M, 96) tile-sorted
    ext = be.unsort_kspace(ks, 0).cpu().numpy().reshape(E, C, -1)
    assert np.all(np.isfinite(ext))
    for e in CHECK_ECHOES:
        ref = cgrid.nufft(img[e][None] * mps, k)                        # (C, M)
        err = onf.rel_l2(ext[e], ref)
        assert err < TOL_NUFFT, (e, err)


def test_adjoint_96_columns_matches_oracle(problem):
    torch, be, k, dcf, mps, img, rng = problem
    M = k.shape[0]
    q = (rng.standard_normal((E, C, M)) + 1j * rng.standard_normal((E, C, M))).astype(np.complex64)
    qs = be.sort_kspace(torch.from_numpy(q.reshape(E * C, M)).cuda(), 0)
    g = be.adjoint_bin(qs, 0, use_dcf=True).cpu().numpy()               # (E, Z, Y, X)
    assert np.all(np.isfinite(g))
    for e in CHECK_ECHOES:
        ref = np.sum(cgrid.nufft_adjoint(dcf * q[e], k, SHAPE) * np.conj(mps), axis=0)
        err = onf.rel_l2(g[e], ref)
        assert err < TOL_NUFFT, (e, err)
    # the gather is deterministic at this size too
    g2 = be.adjoint_bin(qs, 0, use_dcf=True)
    assert torch.equal(g2, be.adjoint_bin(qs, 0, use_dcf=True))


@pytest.mark.parametrize("shape,E,C", [(SHAPE, E, C), ((96, 128, 128), 4, 8)])
def test_fused_yz_passes_equal_the_separate_passes(shape, E, C):
    """The fused y + z kernels (one thread-block cluster per (x, 4-column) plane,
    the intermediate volume in distributed shared memory) run each line through
    the same butterflies as the separate passes: the NUFFT results are equal
    bit for bit.  Shapes: the benchmark's (16-CTA clusters) and the 128x128x96
    TVME workload's (8-CTA clusters).  Plans use them only when asked
    (fuse_yz=True, TR_PLAN_YZ_FUSION): they measured slower than the separate
    passes."""
    torch = _torch()
    syn = pkg("synthetic")
    nb = pkg("nufft_backend")
    rng = np.random.default_rng(11)
    k = syn.cones_trajectory(shape, 512, 300, rng)[:48].reshape(-1, 3)
    dcf = syn.density(k, shape)
    mps = syn.coil_maps(shape, C, rng)
    img = torch.randn((E,) + shape, dtype=torch.complex64, device="cuda")
    q = torch.randn((k.shape[0], E * C), dtype=torch.complex64, device="cuda")
    outs = []
    for fuse in (True, False):
        be = nb.B200NufftBackend(shape, [k], 0, dcf=[dcf], n_coils=C, n_echoes=E, fuse_yz=fuse)
        be.set_maps(mps)
        prof = be.profile(0, reps=1)
        assert ("fwd_yz" in prof and "adj_zy" in prof) == fuse      # the fused kernels ran when allowed
        outs.append((be.forward_bin(img, 0).clone(), be.adjoint_bin(q, 0, use_dcf=True).clone()))
        be.close()
    torch.cuda.synchronize()
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("C,E", [(8, 2), (16, 3)])
def test_two_pass_320_transforms_match_three_pass(C, E):
    """The 320-point FFT passes (here the x passes, k_fwd_x_wide / k_adj_x_wide,
    and the y passes, k_line_tma with radix plan 1) run in two shared-memory
    passes (radices 20 x 16) unless TR_PLAN_THREE_PASS_320 asks for the three of
    the other lengths (5, 8, 8).  Both are the same DFT in a different order of
    float operations: results agree to float rounding (and differ in bits, so
    the flag does select other kernels), and the two-pass ones match the oracle
    at the NUFFT bar."""
    torch = _torch()
    syn = pkg("synthetic")
    nb = pkg("nufft_backend")
    rng = np.random.default_rng(23)
    shape = (16, 256, 256)                                         # OSY = OSX = 320
    k = syn.cones_trajectory(shape, 256, 200, rng)[:40].reshape(-1, 3)
    dcf = syn.density(k, shape)
    mps = syn.coil_maps(shape, C, rng)
    img = (rng.standard_normal((E,) + shape) + 1j * rng.standard_normal((E,) + shape)).astype(np.complex64)
    q = (rng.standard_normal((E * C, k.shape[0])) + 1j * rng.standard_normal((E * C, k.shape[0]))).astype(np.complex64)
    outs = []
    for three in (False, True):
        be = nb.B200NufftBackend(shape, [k], 0, dcf=[dcf], n_coils=C, n_echoes=E, three_pass_320=three)
        be.set_maps(mps)
        assert be.os_shape[1:] == (320, 320)
        fwd = be.unsort_kspace(be.forward_bin(torch.from_numpy(img).cuda(), 0), 0).cpu().numpy()
        adj = be.adjoint_bin(be.sort_kspace(torch.from_numpy(q).cuda(), 0), 0, use_dcf=True).cpu().numpy()
        outs.append((fwd.reshape(E, C, -1), adj))
        be.close()
    (f2, a2), (f3, a3) = outs
    assert onf.rel_l2(f2, f3) < 1e-6 and onf.rel_l2(a2, a3) < 1e-6
    assert not (np.array_equal(f2, f3) and np.array_equal(a2, a3))
    for e in range(E):
        assert onf.rel_l2(f2[e], cgrid.nufft(img[e][None] * mps, k)) < TOL_NUFFT
        ref = np.sum(cgrid.nufft_adjoint(dcf * q.reshape(E, C, -1)[e], k, shape) * np.conj(mps), axis=0)
        assert onf.rel_l2(a2[e], ref) < TOL_NUFFT


@pytest.mark.parametrize("shape,cones,E,C", [((64, 96, 96), 64, 2, 8), ((16, 20, 24), 24, 2, 8), ((16, 20, 24), 24, 2, 3)])
def test_empty_column_skip_gives_the_same_bits(shape, cones, E, C):
    """The z passes leave out the grid lines of (y, x) tile columns that no
    sample's kernel reaches: forward, interpolation never reads them; adjoint,
    gridding writes no tile there and the pass writes their zeros.  On a
    trajectory that leaves most columns empty (64 cones of the benchmark's
    4096) the NUFFT results equal those of a plan that transforms every line
    (TR_PLAN_NO_COLUMN_SKIP) bit for bit, and the per-stage bytes count only
    the occupied lines.  Cases: the compiled z length (TMA pass), a runtime-
    radix one (odd grid, 20 x 25 x 30), and a column count (6) that is not a
    multiple of the z pass's 16 lines per CTA, where a CTA would mix occupied
    and unoccupied columns and the plan does not skip."""
    torch = _torch()
    syn = pkg("synthetic")
    nb = pkg("nufft_backend")
    rng = np.random.default_rng(31)
    k = syn.cones_trajectory(shape, 4096, 300, rng)[:cones].reshape(-1, 3)
    dcf = syn.density(k, shape)
    mps = syn.coil_maps(shape, C, rng)
    img = torch.randn((E,) + shape, dtype=torch.complex64, device="cuda")
    q = torch.randn((k.shape[0], E * C), dtype=torch.complex64, device="cuda")
    outs, prof = [], []
    for skip in (True, False):
        be = nb.B200NufftBackend(shape, [k], 0, dcf=[dcf], n_coils=C, n_echoes=E, column_skip=skip)
        be.set_maps(mps)
        prof.append(be.profile(0, reps=1))
        outs.append((be.forward_bin(img, 0).clone(), be.adjoint_bin(q, 0, use_dcf=True).clone()))
        be.close()
    torch.cuda.synchronize()
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])
    if (E * C) % 16 == 0:
        assert prof[0]["fwd_z"]["bytes"] < prof[1]["fwd_z"]["bytes"]
        assert prof[0]["adj_z"]["bytes"] < prof[1]["adj_z"]["bytes"]
    else:
        assert prof[0]["fwd_z"]["bytes"] == prof[1]["fwd_z"]["bytes"]
