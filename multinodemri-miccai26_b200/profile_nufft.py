"""Per-stage timing of the b200 NUFFT on one bin (CUDA events), for roofline work.

    python multinodemri-miccai26_b200/profile_nufft.py --shape 96 128 128 --coils 16 --echoes 2 --reps 3

Builds one bin of the synthetic cones trajectory (``--cones`` interleaves of
``--readout`` points), random coil maps, and runs ``B200NufftBackend.profile``:
each of the eight batched-NUFFT stages (forward x / y / z passes,
interpolation with the fused dual prox, gridding, adjoint z / y / x passes)
once as warm-up and ``--reps`` times timed.  Prints one JSON line with ms,
algorithmic bytes and GB/s per stage.  Small shapes keep ``ncu --set full``
captures to a few GB of device memory.
"""

from __future__ import annotations

import argparse
import importlib
import json
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))
PKG = Path(__file__).resolve().parent.name


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", type=int, nargs=3, default=[96, 128, 128])
    ap.add_argument("--coils", type=int, default=16)
    ap.add_argument("--echoes", type=int, default=2)
    ap.add_argument("--cones", type=int, default=700)
    ap.add_argument("--readout", type=int, default=600)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--pdhg", type=int, default=0, help="also run this many TVME iterations (all bins)")
    ap.add_argument("--bins", type=int, default=2)
    ap.add_argument("--no-tma", action="store_true", help="stage the FFT passes with cp.async instead of TMA")
    ap.add_argument("--fuse-yz", action="store_true", help="also time the fused y + z cluster kernels")
    ap.add_argument("--three-pass-320", action="store_true",
                    help="run the 320-point transforms in three shared-memory passes (radices 5, 8, 8)")
    ap.add_argument("--no-column-skip", action="store_true",
                    help="transform the z lines of (y, x) tile columns that no sample reaches as well")
    ap.add_argument("--autotune", action="store_true", help="let the plan time its launch-shape candidates")
    args = ap.parse_args(argv)
    import torch
    syn = importlib.import_module(f"{PKG}.synthetic")
    nb = importlib.import_module(f"{PKG}.nufft_backend")
    shape = tuple(args.shape)
    rng = np.random.default_rng(0)
    coord = syn.cones_trajectory(shape, args.cones, args.readout, rng).reshape(-1, 3)
    dcf = syn.density(coord, shape)
    be = nb.B200NufftBackend(shape, [coord], 0, dcf=[dcf], n_coils=args.coils, n_echoes=args.echoes,
                             tma=not args.no_tma, autotune=args.autotune, fuse_yz=args.fuse_yz,
                             three_pass_320=args.three_pass_320, column_skip=not args.no_column_skip)
    mps = syn.coil_maps(shape, args.coils, rng)
    be.set_maps(mps)
    prof = be.profile(0, reps=args.reps)
    torch.cuda.synchronize()
    out = {"tma": not args.no_tma, "spread_columns": be.spread_columns, "shape_zyx": list(shape),
           "os_shape": list(be.os_shape), "coils": args.coils, "echoes": args.echoes, "samples": int(coord.shape[0]), "stages": {k: {kk: round(vv, 4) for kk, vv in v.items()}
                                                      for k, v in prof.items()}}
    be.close()
    if args.pdhg:
        solver = importlib.import_module(f"{PKG}.solver")
        cfg = syn.SyntheticConfig("profile", shape, args.coils, args.echoes, args.bins, args.cones * args.bins,
                                  args.readout, algorithm="tvme")
        ds = syn.make_geometry(cfg)
        syn.simulate_kspace_b200(ds, 0)
        s = solver.PdhgSolver("tvme", shape, [ds.coord[ds.bin_indices(b)] for b in range(args.bins)], ds.bin_dcf(),
                              ds.mps, ds.bin_ksp())
        s.reset()
        s.iterate(1, tol=0.0)
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(s.stream)
        s.iterate(args.pdhg, tol=0.0)
        stop.record(s.stream)
        stop.synchronize()
        out["pdhg_ms_per_iteration"] = round(start.elapsed_time(stop) / args.pdhg, 4)
        out["pdhg_bins"] = args.bins
        s.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
