"""GPU PDHG (TVM / TVME / TVMW) against the golden vectors of the reference reconstructors."""

import numpy as np
import pytest

from _fixtures import binned, load_golden, oracle_problem, pkg
from oracle import nufft as onf
from oracle import pdhg as op

pytestmark = pytest.mark.gpu

TOL_PDHG = 1e-3    # north-star bar vs the reference PDHG image at equal iteration count


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _solver(fx, use_graph=True):
    solver = pkg("solver")
    coords, dcfs, ksps = binned(fx)
    shape = tuple(int(v) for v in fx["shape"])
    lam = float(fx["lam"])
    return solver.PdhgSolver(str(fx["alg"]), shape, coords, dcfs, fx["mps"], ksps, l2_coupling=bool(fx["l2"]),
                             lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam, use_graph=use_graph)


@pytest.mark.parametrize("name", ["tvm", "tvm_l2", "tvme", "tvme_l2", "tvmw"])
def test_pdhg_k_iterations_match_reference(name):
    _torch()
    fx = load_golden(name)
    s = _solver(fx)
    r = s.run(max_iter=int(fx["n_iter"]), tol=0.0)
    assert r.iterations == int(fx["n_iter"])
    err = onf.rel_l2(r.image.cpu().numpy(), fx["image_k"])
    assert err < 1e-4, err
    s.close()


@pytest.mark.parametrize("name", ["tvm", "tvme", "tvme_l2", "tvmw"])
def test_pdhg_stopping_rule_matches_reference(name):
    _torch()
    fx = load_golden(name)
    s = _solver(fx)
    r = s.run(max_iter=60, tol=float(fx["tol_stop"]))
    assert r.iterations == int(fx["iters_tol"])
    assert onf.rel_l2(r.image.cpu().numpy(), fx["image_tol"]) < TOL_PDHG
    s.close()


def test_graph_replay_equals_eager():
    torch = _torch()
    fx = load_golden("tvme")
    a = _solver(fx, use_graph=True)
    b = _solver(fx, use_graph=False)
    ra = a.run(max_iter=6, tol=0.0).image.clone()
    rb = b.run(max_iter=6, tol=0.0).image.clone()
    assert torch.equal(ra, rb)
    a.close()
    b.close()


def test_fp64_oracle_equal_iterations():
    """b200 float32 vs the FP64 PDHG oracle after 12 iterations (TVME, L2 coupling)."""
    _torch()
    fx = load_golden("tvme_l2")
    s = _solver(fx)
    r = s.run(max_iter=12, tol=0.0)
    lam = float(fx["lam"])
    ref = op.run("tvme", oracle_problem(fx, np.complex128), max_iter=12, tol=0.0, lam_m=lam, lam_e=lam,
                 l2_coupling=True)
    assert onf.rel_l2(r.image.cpu().numpy(), ref.image) < TOL_PDHG
    s.close()
