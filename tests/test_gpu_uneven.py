"""Uneven motion bins (Dirichlet(2) bin sizes, the batched-uneven workload's
binning) on the GPU solver against the FP64 PDHG oracle, single plan and
bin-sharded with copied halos."""

from dataclasses import replace

import numpy as np
import pytest

from _fixtures import pkg
from oracle import nufft as onf
from oracle import pdhg as op

pytestmark = pytest.mark.gpu


def _problem():
    syn = pkg("synthetic")
    cfg = replace(syn.scaled(syn.CONFIGS["tvme-256-dirichlet"], 0.125), n_coils=4, n_echoes=2, seed=5)
    ds = syn.make_geometry(cfg)
    syn.simulate_kspace_b200(ds, 0)
    coords = [ds.coord[ds.bin_indices(b)].reshape(-1, 3) for b in range(cfg.n_bins)]
    dcfs = [d.reshape(-1) for d in ds.bin_dcf()]
    ksps = [k.reshape(k.shape[0], k.shape[1], -1) for k in ds.bin_ksp()]
    return cfg, ds, coords, dcfs, ksps


def test_dirichlet_bins_match_fp64_oracle():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    solver = pkg("solver")
    cfg, ds, coords, dcfs, ksps = _problem()
    counts = [c.shape[0] for c in coords]
    assert len(set(counts)) > 1 and min(counts) > 0          # genuinely uneven bins
    n_iter = 3
    s = solver.PdhgSolver("tvme", cfg.img_shape, coords, dcfs, ds.mps, ksps, lam_m=cfg.lam, lam_e=cfg.lam)
    got = s.run(max_iter=n_iter, tol=0.0).image.cpu().numpy()
    s.close()
    pb = op.Problem(nufft=op.OracleNufft(cfg.img_shape, coords), ksp=ksps, dcf=dcfs, mps=ds.mps)
    ref = op.run("tvme", pb, max_iter=n_iter, tol=0.0, lam_m=cfg.lam, lam_e=cfg.lam)
    err = onf.rel_l2(got, ref.image)
    assert err < 1e-3, err


def test_dirichlet_bins_sharded_equal_single_plan():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    solver, par = pkg("solver"), pkg("parallel")
    cfg, ds, coords, dcfs, ksps = _problem()
    counts = [c.shape[0] for c in coords]
    ranges = par.partition_bins(counts, 3)
    whole = solver.PdhgSolver("tvme", cfg.img_shape, coords, dcfs, ds.mps, ksps, lam_m=cfg.lam, lam_e=cfg.lam)
    ref = whole.run(max_iter=4, tol=0.0).image.clone()
    sv = [solver.PdhgSolver("tvme", cfg.img_shape, coords[a:e], dcfs[a:e], ds.mps, ksps[a:e], lam_m=cfg.lam,
                            lam_e=cfg.lam) for a, e in ranges]
    eng = [par.B200ShardEngine(s, a, len(counts)) for s, (a, e) in zip(sv, ranges)]
    for en in eng:
        en.reset(None)
    for _ in range(4):
        for r in range(len(eng) - 1):
            eng[r].u_bar_next.copy_(eng[r + 1].first_u_bar())
        for en in eng:
            en.phase1(1 / 6, 1 / 6)
        for r in range(1, len(eng)):
            eng[r].p_m_prev.copy_(eng[r - 1].last_p_m())
        for en in eng:
            en.phase2(1 / 6, 1 / 6)
    img = torch.cat([en.image() for en in eng])
    torch.cuda.synchronize()
    assert torch.equal(img, ref)
    for s in sv + [whole]:
        s.close()
