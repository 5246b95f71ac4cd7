"""The power-iteration step rule and the bounded-wait error path on the GPU.

* ``tr_power_iteration`` (FP64 norms of the batched data operator
  A^H W A) against the oracle's FP64 power iteration;
* a solve with the power rule's block-diagonal steps against the FP64 PDHG
  oracle run with the same steps (equal iteration count, 1e-3);
* a fixed point of one step rule is a fixed point of the other: both rules
  solve the same saddle-point problem, so one reference-rule iteration from a
  state the power rule has settled moves it no more than the power rule does;
* ``tr_plan_set_wait_limit(0)``: every bounded TMA wait gives up at once, the
  copies in flight still land, and the solve reports ``TR_ERR_TIMEOUT``; with
  the default limit restored the same plan gives the same bits as a fresh one.
"""

import numpy as np
import pytest

from _fixtures import binned, load_golden, oracle_problem, pkg
from oracle import cgrid
from oracle import nufft as onf
from oracle import pdhg as op

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _solver(fx, **kw):
    solver = pkg("solver")
    coords, dcfs, ksps = binned(fx)
    lam = float(fx["lam"])
    return solver.PdhgSolver(str(fx["alg"]), tuple(int(v) for v in fx["shape"]), coords, dcfs, fx["mps"], ksps,
                             l2_coupling=bool(fx["l2"]), lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam, **kw)


@pytest.mark.parametrize("name", ["tvme", "tvmw"])
def test_power_norm_matches_fp64_oracle(name):
    _torch()
    fx = load_golden(name)
    s = _solver(fx)
    got = s.backend.power_norm(n_iter=80, seed=3)
    ref = op.power_norm(oracle_problem(fx), n_iter=80, seed=3)
    s.close()
    assert abs(got - ref) <= 1e-3 * ref, (got, ref)


@pytest.mark.parametrize("name", ["tvm", "tvme", "tvmw"])
def test_power_rule_solve_matches_fp64_oracle(name):
    _torch()
    fx = load_golden(name)
    s = _solver(fx, step_rule="power", power_iters=60)
    assert s.step_rule == "power" and s.data_norm > 0
    r = s.run(max_iter=12, tol=0.0)
    assert (r.sigma, r.tau, r.sigma_data) == (s.sigma, s.tau, s.sigma_data)
    lam = float(fx["lam"])
    ref = op.run(name, oracle_problem(fx), max_iter=12, tol=0.0, sigma=r.sigma, tau=r.tau, sigma_data=r.sigma_data,
                 lam_m=lam, lam_e=lam, lam1=lam, lam2=lam, lam3=lam, l2_coupling=bool(fx["l2"]))
    err = onf.rel_l2(r.image.cpu().numpy(), ref.image)
    s.close()
    assert err < 1e-3, err


def test_power_rule_reaches_the_reference_rule_fixed_point():
    """Both rules solve the same saddle-point problem, so they share its fixed
    point.  On a small well-posed TVM problem (random samples at 1.3x the voxel
    count per coil, two coils, lambda 1e-9) both settle: the power rule within
    600 iterations, the reference's sigma = tau = 1/6 within 3000."""
    _torch()
    syn = pkg("synthetic")
    solver = pkg("solver")
    shape = (12, 16, 16)
    rng = np.random.default_rng(1)
    coords = [np.stack([rng.uniform(-n / 2, n / 2, 4000) for n in shape], -1).astype(np.float32) for _ in range(2)]
    dcfs = [syn.density(c, shape) for c in coords]
    mps = syn.coil_maps(shape, 2, rng)
    truth = rng.standard_normal((2, 1) + shape) + 1j * rng.standard_normal((2, 1) + shape)
    ksps = [cgrid.nufft((truth[b][:, None] * mps[None]).astype(np.complex64), coords[b]) for b in range(2)]
    a = solver.PdhgSolver("tvm", shape, coords, dcfs, mps, ksps, lam_m=1e-9, step_rule="power", power_iters=60)
    ra = a.run(max_iter=600, tol=0.0)
    b = solver.PdhgSolver("tvm", shape, coords, dcfs, mps, ksps, lam_m=1e-9)
    rb = b.run(max_iter=3000, tol=0.0)
    assert ra.tols[-1] < 1e-5 and rb.tols[-1] < 1e-5, (ra.tols[-1], rb.tols[-1])
    err = onf.rel_l2(ra.image.cpu().numpy(), rb.image.cpu().numpy())
    a.close()
    b.close()
    assert err < 1e-3, err


def test_timeout_path_reports_and_recovers():
    torch = _torch()
    syn = pkg("synthetic")
    solver = pkg("solver")
    lib = pkg("_lib")
    # a geometry whose FFT passes and gridding take the TMA paths (compiled
    # lengths 60 and 80, an even column count)
    shape = (48, 64, 64)
    rng = np.random.default_rng(4)
    coords = [syn.cones_trajectory(shape, 40, 120, rng).reshape(-1, 3) for _ in range(2)]
    dcfs = [syn.density(c, shape) for c in coords]
    mps = syn.coil_maps(shape, 4, rng)
    ksps = [(rng.standard_normal((2, 4, c.shape[0])) + 1j * rng.standard_normal((2, 4, c.shape[0])))
            .astype(np.complex64) for c in coords]

    def make():
        return solver.PdhgSolver("tvme", shape, coords, dcfs, mps, ksps)

    a = make()
    a.backend.set_wait_limit(0)
    with pytest.raises(lib.TrError) as exc:
        a.run(max_iter=3, tol=0.0)
    assert exc.value.code == lib.TR_ERR_TIMEOUT
    assert "bounded device wait" in str(exc.value)
    a.backend.set_wait_limit()                          # default limit: the context is still usable
    ra = a.run(max_iter=3, tol=0.0).image.clone()
    b = make()
    rb = b.run(max_iter=3, tol=0.0).image.clone()
    torch.cuda.synchronize()
    assert torch.equal(ra, rb)
    a.close()
    b.close()


def test_power_iteration_rejects_a_zero_start():
    torch = _torch()
    fx = load_golden("tvm")
    s = _solver(fx)
    lib = pkg("_lib")
    with pytest.raises(ValueError, match="zero"):
        s.backend.power_norm(n_iter=2, work=torch.zeros((s.B,) + s.img_shape, dtype=torch.complex64,
                                                        device=s.device))
    s.close()
