"""What the trained warm-start network gains over the zero start (held-out phantom).

Both solves run the same PDHG iterations; the warm one starts from the
network's estimate (with the data dual at its fixed-point relation).  A long
zero-start solve stands in for the PDHG fixed point; after a fixed iteration
budget the warm-started iterate must be closer to it than the plain one.
"""

from dataclasses import replace

import pytest

from _fixtures import pkg

pytestmark = pytest.mark.gpu


def test_trained_network_gains_over_zero_start():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    syn, solver, ws = pkg("synthetic"), pkg("solver"), pkg("warmstart")
    net = ws.load_model()
    cfg = replace(syn.CONFIGS["warm-96"], seed=4242)           # not among the training seeds (1000..1033)
    ds = syn.make_geometry(cfg)
    syn.simulate_kspace_b200(ds, 0)
    s = solver.PdhgSolver(cfg.algorithm, cfg.img_shape, [ds.coord[ds.bin_indices(b)] for b in range(cfg.n_bins)],
                          ds.bin_dcf(), ds.mps, ds.bin_ksp(), lam_m=cfg.lam, lam_e=cfg.lam)
    ref = s.run(max_iter=800, tol=0.0).image.clone()
    rel = lambda a: float((a - ref).norm() / ref.norm())
    out = {}
    for k in (30, 100):
        plain = rel(s.run(max_iter=k, tol=0.0).image)
        warm = rel(ws.warm_solve(s, cfg, max_iter=k, tol=0.0, model=net).image)
        out[k] = (plain, warm)
    s.close()
    print("distance to the 800-iteration solve (plain, warm):", out)
    for k, (plain, warm) in out.items():
        assert warm < plain, (k, plain, warm)
