"""Bin-sharded PDHG kernels on one GPU: two shards driven in one process.

``tr_pdhg_phase`` with halos must reproduce the single-plan iteration: the
two halves of the golden problems' bins run as two plans whose halos (u_bar
forward, p_m backward) are copied between them in this process, with no
cross-shard waiting on the device, and the summed stopping sums are the whole
problem's.  The multi-process NCCL path uses the same engine and phases; its
orchestration is covered over gloo in test_parallel_cpu.py.
"""

import numpy as np
import pytest

from _fixtures import binned, load_golden, pkg

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _solver(fx, sl=slice(None)):
    solver = pkg("solver")
    coords, dcfs, ksps = binned(fx)
    shape = tuple(int(v) for v in fx["shape"])
    lam = float(fx["lam"])
    return solver.PdhgSolver(str(fx["alg"]), shape, coords[sl], dcfs[sl], fx["mps"], ksps[sl],
                             l2_coupling=bool(fx["l2"]), lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam)


@pytest.mark.parametrize("name", ["tvm", "tvme", "tvme_l2", "tvmw"])
def test_two_shards_equal_one_plan(name):
    torch = _torch()
    par = pkg("parallel")
    fx = load_golden(name)
    nb = len(binned(fx)[0])
    cut = nb // 2 if nb > 2 else 1
    whole = _solver(fx)
    ref = whole.run(max_iter=5, tol=0.0)
    ref_img = ref.image.clone()
    s0, s1 = _solver(fx, slice(0, cut)), _solver(fx, slice(cut, None))
    e0 = par.B200ShardEngine(s0, 0, nb)
    e1 = par.B200ShardEngine(s1, cut, nb)
    e0.reset(None)
    e1.reset(None)
    tols = []
    for _ in range(5):
        # shard 0 runs phase 1 in its two parts (3: local state, 4: with the halo), as the
        # sharded loop does with the halo in flight in between; shard 1 runs it whole
        e0.phase1a(1 / 6, 1 / 6)
        e0.u_bar_next.copy_(e1.first_u_bar())
        e0.phase1b(1 / 6, 1 / 6)
        e1.phase1(1 / 6, 1 / 6)
        e1.p_m_prev.copy_(e0.last_p_m())
        sums = e0.phase2(1 / 6, 1 / 6) + e1.phase2(1 / 6, 1 / 6)
        num, den = (float(v) for v in sums.tolist())
        tols.append(par.tolerance_from(name, num, den))
    img = torch.cat([e0.image(), e1.image()])
    torch.cuda.synchronize()
    # same kernels and per-element arithmetic: the images agree bit for bit
    assert torch.equal(img, ref_img)
    np.testing.assert_allclose(tols, ref.tols, rtol=1e-9)
    for s in (whole, s0, s1):
        s.close()


def test_phase_rejects_missing_halo():
    _torch()
    par = pkg("parallel")
    lib = pkg("_lib")
    fx = load_golden("tvme")
    nb = len(binned(fx)[0])
    s0 = _solver(fx, slice(0, 1))
    e0 = par.B200ShardEngine(s0, 0, nb)
    e0.reset(None)
    e0.shard.u_bar_next = None           # the plan does not hold the last bin: the halo is required
    with pytest.raises(ValueError, match="u_bar_next"):
        e0.phase1(1 / 6, 1 / 6)
    s0.close()
    assert lib.TR_ERR_INVALID_ARG == 1
