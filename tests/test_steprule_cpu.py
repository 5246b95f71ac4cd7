"""Host-side checks of the PDHG step rules (no GPU).

* ``power_steps`` satisfies the block-diagonal PDHG bound
  tau (sigma_data ||A||^2 + sigma ||K_reg||^2) < 1;
* ``REG_NORM2`` bounds the regulariser operators of each algorithm, by
  power iteration on K^T K with the oracle's operators and their transposes;
* the oracle's FP64 power iteration (the GPU test's checker) finds the largest
  eigenvalue of an explicitly assembled A^H W A;
* ``PdhgSolver.run`` retries a non-finite solve with every step scaled by 0.9
  (``tvme.py:571-573``) and re-raises for TVMW, whose reference has no retry.
"""

import math

import numpy as np
import pytest

from _fixtures import pkg
from oracle import nufft as onf
from oracle import pdhg as op
from oracle import wavelets as ow


@pytest.mark.parametrize("alg", ["tvm", "tvme", "tvmw"])
@pytest.mark.parametrize("norm", [0.05, 0.2, 1.0, 7.5])
def test_power_steps_satisfy_the_block_bound(alg, norm):
    solver = pkg("solver")
    sigma, tau, sigma_data = solver.power_steps(alg, norm)
    total = tau * (sigma_data * norm * norm + sigma * solver.REG_NORM2[alg])
    assert 0.98 < total < 1.0
    assert sigma > 0 and tau > 0 and sigma_data == 0.1
    with pytest.raises(ValueError):
        solver.power_steps(alg, 0.0)
    with pytest.raises(ValueError):
        solver.power_steps("tv", norm)


def _reg_normal(alg, x):
    """K_reg^T K_reg x with the oracle's operators (x: (B, E, Z, Y, X))."""
    dm = op.motion_diff(x)
    if alg == "tvm":
        return op.motion_div_tvme(dm)
    if alg == "tvme":
        de = np.zeros_like(x)
        de[:, :-1] = x[:, 1:] - x[:, :-1]
        spatial = op.dxb(op.dxf(de)) + op.dyb(op.dyf(de)) + op.dzb(op.dzf(de))
        return op.motion_div_tvme(dm) + op.echo_div_tvme(spatial)
    w2 = np.stack([np.stack([ow.waverec3(ow.wavedec3(x[b, e], "db6"), "db6")[tuple(slice(0, n) for n in x.shape[2:])]
                             for e in range(x.shape[1])]) for b in range(x.shape[0])])
    return op.motion_div_tvme(dm) + ow.w1_adjoint(ow.w1_forward(x)) + w2


@pytest.mark.parametrize("alg,shape", [("tvm", (4, 1, 6, 8, 8)), ("tvme", (4, 4, 6, 8, 8)),
                                       ("tvmw", (3, 3, 24, 24, 24))])
def test_regulariser_norm_bounds(alg, shape):
    solver = pkg("solver")
    rng = np.random.default_rng(0)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = 0.0
    for _ in range(150):
        x /= np.linalg.norm(x.ravel())
        x = _reg_normal(alg, x)
        lam = float(np.linalg.norm(x.ravel()))
    assert lam <= solver.REG_NORM2[alg] * (1 + 1e-9), lam


def test_motion_and_echo_transposes():
    """The oracle's divergences are the exact transposes of its differences."""
    rng = np.random.default_rng(1)
    x = rng.standard_normal((3, 4, 5, 6, 7))
    p = rng.standard_normal((3, 4, 5, 6, 7))
    assert np.vdot(op.motion_diff(x), p) == pytest.approx(np.vdot(x, op.motion_div_tvme(p)))
    de = np.zeros_like(x)
    de[:, :-1] = x[:, 1:] - x[:, :-1]
    assert np.vdot(de, p) == pytest.approx(np.vdot(x, op.echo_div_tvme(p)))
    for f, b in ((op.dxf, op.dxb), (op.dyf, op.dyb), (op.dzf, op.dzb)):
        assert np.vdot(f(x), p) == pytest.approx(np.vdot(x, b(p)))


def test_oracle_power_norm_finds_the_largest_eigenvalue():
    shape = (4, 5, 6)
    rng = np.random.default_rng(2)
    coords = [np.stack([rng.uniform(-n / 2, n / 2, 40) for n in shape], -1).astype(np.float32)]
    dcf = [rng.uniform(0.2, 1.0, 40)]
    mps = (rng.standard_normal((2,) + shape) + 1j * rng.standard_normal((2,) + shape))
    pb = op.Problem(op.OracleNufft(shape, coords), [np.zeros((1, 2, 40), np.complex128)], dcf, mps)
    pb.cast()
    n = int(np.prod(shape))
    mat = np.zeros((n, n), dtype=np.complex128)
    for i in range(n):
        e = np.zeros(n, dtype=np.complex128)
        e[i] = 1.0
        img = e.reshape((1, 1) + shape)
        ksp = [pb.nufft.forward(img[0][:, None] * pb.mps[None], 0)]
        mat[:, i] = op.data_grad(pb, ksp).ravel()
    assert np.allclose(mat, mat.conj().T, atol=1e-10)          # A^H W A is Hermitian
    lam_max = float(np.linalg.eigvalsh(mat).max())
    assert op.power_norm(pb, n_iter=300) == pytest.approx(math.sqrt(lam_max), rel=1e-6)


class _FakeEvent:
    def __init__(self, enable_timing=True):
        pass

    def record(self, stream=None):
        pass

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return 1.0


class _FakeTorch:
    class cuda:
        Event = _FakeEvent


@pytest.mark.parametrize("alg,retries", [("tvme", 2), ("tvm", 1)])
def test_overflow_retry_shrinks_every_step(alg, retries):
    solver = pkg("solver")
    lib = pkg("_lib")
    s = solver.PdhgSolver.__new__(solver.PdhgSolver)
    s.torch, s.algorithm, s.stream = _FakeTorch, alg, None
    s.sigma, s.tau, s.sigma_data = 0.5, 2.0, 0.25
    s.step_rule, s.data_norm, s.setup_seconds = "power", 1.0, 0.0
    s.u_bar = "image"
    calls = []

    def iterate(n, tol, sigma, tau, sigma_data):
        calls.append((sigma, tau, sigma_data))
        if len(calls) <= retries:
            raise lib.TrNonFinite(lib.TR_ERR_NONFINITE, "non-finite value")
        return 5, [1.0, 0.5]

    s.reset = lambda init=None: None
    s.iterate = iterate
    r = s.run(max_iter=10, tol=1e-3)
    assert len(calls) == retries + 1
    for k, (sg, ta, sd) in enumerate(calls):
        assert (sg, ta, sd) == pytest.approx((0.5 * 0.9 ** k, 2.0 * 0.9 ** k, 0.25 * 0.9 ** k))
    assert (r.sigma, r.tau, r.sigma_data) == pytest.approx(calls[-1])
    assert r.iterations == 5 and r.image == "image"


def test_overflow_is_not_retried_for_tvmw():
    solver = pkg("solver")
    lib = pkg("_lib")
    s = solver.PdhgSolver.__new__(solver.PdhgSolver)
    s.torch, s.algorithm, s.stream = _FakeTorch, "tvmw", None
    s.sigma = s.tau = s.sigma_data = 1 / 6
    s.step_rule, s.data_norm, s.setup_seconds = "reference", None, 0.0
    s.reset = lambda init=None: None

    def iterate(*a):
        raise lib.TrNonFinite(lib.TR_ERR_NONFINITE, "non-finite value")

    s.iterate = iterate
    with pytest.raises(OverflowError):
        s.run(max_iter=10)
