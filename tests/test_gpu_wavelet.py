"""GPU parity of the TVMW spatial wavelet (db6, zero mode) at three levels.

The TVMW workload (160 x 160 x 112) decomposes to PyWavelets' maximum level
3; a 112 x 96 x 96 image does too (and its 1.25x grid, 140 x 120 x 120,
factors into the NUFFT's radices), so these cases run the level-to-level
hand-off of csrc/tr_wavelet.cu (the approximation of level l becoming the
input of level l + 1, the detail offsets of every level, and the synthesis
crop to the next finer level's length) that the one-level golden fixtures do
not reach.  Reference: ptwt wavedec3 / waverec3 (tvmw.py:196-206) and the
TVMW iteration (tvmw.py:385-685), against the oracle's restatement.
"""

import numpy as np
import pytest

from _fixtures import pkg
from oracle import cgrid
from oracle import nufft as onf
from oracle import pdhg as op
from oracle import wavelets as ow

pytestmark = pytest.mark.gpu

SHAPE = (112, 96, 96)
TOL_WAVELET = 1e-5


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _flatten(tree) -> np.ndarray:
    """wavedec3 list of one image -> [cA_L | 7 bands of level L | ... | level 1]."""
    parts = [tree[0].ravel()]
    for level in tree[1:]:
        parts.extend(level[key].ravel() for key in ow.DETAIL_KEYS)
    return np.concatenate(parts)


def _unflatten(flat: np.ndarray, shape) -> list:
    shapes = ow.coeff_shapes(shape, "db6")
    pos = 0
    n0 = int(np.prod(shapes[0]))
    tree = [flat[:n0].reshape(shapes[0])]
    pos = n0
    for s in shapes:
        n = int(np.prod(s))
        level = {}
        for key in ow.DETAIL_KEYS:
            level[key] = flat[pos:pos + n].reshape(s)
            pos += n
        tree.append(level)
    assert pos == flat.size
    return tree


@pytest.fixture(scope="module")
def backend():
    torch = _torch()
    nb = pkg("nufft_backend")
    rng = np.random.default_rng(11)
    k = np.stack([rng.uniform(-n / 2, n / 2, 500) for n in SHAPE], -1).astype(np.float32)
    be = nb.B200NufftBackend(SHAPE, [k, k], 0, n_coils=1, n_echoes=2)     # B = 2, E = 2: four images
    assert be.wavelet_levels == 3 == ow.max_level(SHAPE, 12)
    yield torch, be, rng
    be.close()


def test_w2_analysis_three_levels_matches_oracle(backend):
    torch, be, rng = backend
    x = (rng.standard_normal((2, 2) + SHAPE) + 1j * rng.standard_normal((2, 2) + SHAPE)).astype(np.complex64)
    c = be.wavelet_forward(torch.from_numpy(x).cuda()).cpu().numpy()          # (4, ncoef)
    assert c.shape == (4, be.wavelet_coeffs)
    for i, img in enumerate(x.reshape((4,) + SHAPE)):
        ref = _flatten(ow.wavedec3(img.astype(np.complex128), "db6"))
        assert ref.size == be.wavelet_coeffs
        assert onf.rel_l2(c[i], ref) < TOL_WAVELET, i


def test_w2_synthesis_three_levels_matches_oracle(backend):
    torch, be, rng = backend
    n = be.wavelet_coeffs
    c = (rng.standard_normal((4, n)) + 1j * rng.standard_normal((4, n))).astype(np.complex64)
    y = be.wavelet_adjoint(torch.from_numpy(c).cuda()).cpu().numpy().reshape((4,) + SHAPE)
    for i in range(4):
        rec = ow.waverec3(_unflatten(c[i].astype(np.complex128), SHAPE), "db6")
        ref = rec[tuple(slice(0, s) for s in SHAPE)]
        assert onf.rel_l2(y[i], ref) < TOL_WAVELET, i


def test_w2_perfect_reconstruction_and_isometry(backend):
    """waverec3(wavedec3(x)) = x and ||wavedec3(x)|| = ||x|| (orthogonal db6 filters,
    zero extension keeps every nonzero coefficient)."""
    torch, be, rng = backend
    x = torch.randn((2, 2) + SHAPE, dtype=torch.complex64, device="cuda")
    c = be.wavelet_forward(x)
    y = be.wavelet_adjoint(c)
    assert float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x)) < 1e-5
    ratio = float(torch.linalg.vector_norm(c) / torch.linalg.vector_norm(x))
    assert abs(ratio - 1.0) < 1e-5


def test_tvmw_pdhg_three_levels_matches_fp64_oracle():
    """Four TVMW iterations at three wavelet levels against the FP64 PDHG oracle
    (the north-star bar at equal iteration count: 1e-3 relative L2)."""
    _torch()
    syn = pkg("synthetic")
    solver = pkg("solver")
    cfg = syn.SyntheticConfig("tvmw-3level", SHAPE, 2, 2, 2, 160, 120, algorithm="tvmw")
    ds = syn.make_geometry(cfg)
    syn.simulate_kspace(ds, lambda imgs, k: cgrid.nufft(imgs, k))
    coords = [ds.coord[ds.bin_indices(b)].reshape(-1, 3) for b in range(cfg.n_bins)]
    dcfs = [ds.dcf[ds.bin_indices(b)].reshape(-1) for b in range(cfg.n_bins)]
    ksps = [ds.ksp[:, :, ds.bin_indices(b)].reshape(cfg.n_echoes, cfg.n_coils, -1) for b in range(cfg.n_bins)]
    lam = 1e-4
    s = solver.PdhgSolver("tvmw", SHAPE, coords, dcfs, ds.mps, ksps, lam_m=lam, lam_w1=lam, lam_w2=lam)
    assert s.backend.wavelet_levels == 3
    r = s.run(max_iter=4, tol=0.0)
    pb = op.Problem(op.OracleNufft(SHAPE, coords), [k.astype(np.complex128) for k in ksps], dcfs, ds.mps)
    ref = op.run("tvmw", pb, max_iter=4, tol=0.0, lam1=lam, lam2=lam, lam3=lam)
    err = onf.rel_l2(r.image.cpu().numpy(), ref.image)
    s.close()
    assert err < 1e-3, err
    assert r.tols == pytest.approx(ref.tols, rel=1e-3)
