"""The CPU oracle against the reference: golden PDHG vectors and NUFFT/wavelet properties."""

import numpy as np
import pytest

from _fixtures import load_golden, oracle_problem
from oracle import nufft as onf
from oracle import pdhg as op
from oracle import wavelets as owv

GOLDEN = ["tvm", "tvm_l2", "tvme", "tvme_l2", "tvmw"]


def _run(fx, dtype, iters, tol):
    lam = float(fx["lam"])
    pb = oracle_problem(fx, dtype)
    return op.run(str(fx["alg"]), pb, max_iter=iters, tol=tol, lam_m=lam, lam_e=lam, lam1=lam,
                  lam2=lam, lam3=lam, l2_coupling=bool(fx["l2"]))


@pytest.mark.parametrize("name", GOLDEN)
def test_pdhg_matches_reference_golden(name):
    """complex64 restatement reproduces the reference reconstructor's u_bar after k iterations."""
    fx = load_golden(name)
    r = _run(fx, np.complex64, int(fx["n_iter"]), 0.0)
    assert onf.rel_l2(r.image, fx["image_k"]) < 1e-6
    r64 = _run(fx, np.complex128, int(fx["n_iter"]), 0.0)
    assert onf.rel_l2(r64.image, fx["image_k"]) < 1e-5


@pytest.mark.parametrize("name", ["tvm", "tvme_l2", "tvmw"])
def test_pdhg_stopping_rule_matches_reference(name):
    fx = load_golden(name)
    r = _run(fx, np.complex128, 60, float(fx["tol_stop"]))
    assert r.iterations == int(fx["iters_tol"])
    assert onf.rel_l2(r.image, fx["image_tol"]) < 1e-5


def _rand_problem(shape, M, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    k = np.stack([rng.uniform(-n / 2, n / 2, M) for n in shape], -1).astype(np.float32)
    k[0] = 0.0
    return x, k, rng


def test_nufft_close_to_direct_nudft():
    x, k, _ = _rand_problem((12, 16, 14), 400, 0)
    err = onf.rel_l2(onf.nufft(x, k), onf.nudft(x, k))
    assert err < 1.2e-2  # intrinsic error of KB width 4 at 1.25x oversampling
    # the same code converges with a wider kernel / more oversampling
    assert onf.rel_l2(onf.nufft(x, k, oversamp=2.0, width=6), onf.nudft(x, k)) < 5e-5


def test_nufft_adjointness():
    x, k, rng = _rand_problem((10, 12, 16), 300, 1)
    y = rng.standard_normal(300) + 1j * rng.standard_normal(300)
    lhs = np.vdot(onf.nufft(x, k), y)
    rhs = np.vdot(x, onf.nufft_adjoint(y, k, x.shape))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_kb_taps_five_at_integer_coordinate():
    beta = onf.kb_beta()
    taps, w = onf._tap_weights(np.array([10.0]), 4, beta)
    assert list(taps[0]) == [8, 9, 10, 11, 12]
    assert np.all(w[0] > 0) and abs(w[0, 0] - 1.0) < 1e-12
    taps, w = onf._tap_weights(np.array([10.25]), 4, beta)
    assert w[0, -1] == 0.0 and np.all(w[0, :4] > 0)


def test_bessel_i0_approximation():
    from math import fsum, factorial
    for x in [0.0, 1.0, 3.7, 3.8, 6.99]:
        exact = fsum((x / 2) ** (2 * m) / factorial(m) ** 2 for m in range(60))
        assert abs(onf.bessel_i0_as(np.array([x]))[0] - exact) < 3e-7 * exact


def test_daubechies_filters_properties():
    for n in (1, 2, 6):
        dl, dh, rl, rh = owv.filter_bank(f"db{n}")
        assert abs(rl.sum() - np.sqrt(2)) < 1e-12
        assert abs(np.dot(rl, rl) - 1) < 1e-12
        for s in range(1, n):  # orthogonality to even shifts
            assert abs(np.dot(rl[2 * s:], rl[:-2 * s])) < 1e-12
        k = np.arange(rh.size)
        for m in range(n):  # vanishing moments of the high-pass
            assert abs(np.sum(rh * k ** m)) < 1e-8 * max(1, rh.size ** m)


@pytest.mark.parametrize("shape", [(48, 64, 64), (30, 40, 36), (24, 24, 22)])
def test_wavelet_perfect_reconstruction(shape):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2,) + shape)
    c = owv.wavedec3(x, "db6")
    assert len(c) - 1 == owv.max_level(shape, 12)
    r = owv.waverec3(c, "db6")
    assert r.shape[1:] == shape
    assert np.abs(r - x).max() < 1e-10


def test_wavelet_levels_of_configs():
    assert owv.coeff_shapes((112, 160, 160)) == [(23, 29, 29), (36, 48, 48), (61, 85, 85)]
    assert owv.coeff_shapes((48, 64, 64)) == [(20, 24, 24), (29, 37, 37)]


def test_w1_adjoint_pair():
    rng = np.random.default_rng(4)
    for E in (1, 2, 3, 6):
        u = rng.standard_normal((2, E, 3, 4, 5)) + 1j * rng.standard_normal((2, E, 3, 4, 5))
        p = rng.standard_normal(u.shape) + 1j * rng.standard_normal(u.shape)
        lhs = np.vdot(owv.w1_forward(u), p)
        rhs = np.vdot(u, owv.w1_adjoint(p))
        assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs))
