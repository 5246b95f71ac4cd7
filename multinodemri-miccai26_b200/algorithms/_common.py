"""Single-rank problem assembly, reconstructors and CLI mains for TVM / TVME / TVMW.

Mirrors, for one device, the reference's ``main`` functions
(``algorithms/tvm.py:494-1088``, ``tvme.py:578-1053``, ``tvmw.py:789-1240``):
the same flags (both spellings), the same data preparation (a14 of the
reference's hot path) and the same outputs, with the PDHG loop replaced by
``PdhgSolver`` (``--nufft-backend b200``).  Preparation, per algorithm:

* coordinates: CFL ``ktraj`` xyz -> zyx, readout fraction, ``coord.max() > 1000``
  guard, ``coord[..., d] *= voxel[d] * n[d]``, FoV scaling (``tvme.py:726-798``);
* TVM / TVME: drop the 2 % respiratory outliers, keep the first
  ``int(TR / acc)`` trajectories (``tvme.py:742-754``); TVMW skips both;
* density: TVME divides by its maximum before binning; TVM before and after;
  TVMW after binning only (``tvme.py:802-804``, ``tvm.py:956-959``,
  ``tvmw.py:1129-1133``);
* bin edges ``percentile(resp, linspace(0, 100, B + 1))`` and the half-open
  selection (``tvme.py:853-881``);
* k-space divided by its maximum magnitude, maps by their root sum of
  squares (TVME clamps at 1e-12, TVM / TVMW map zero to one; ``tvme.py:937-949``).
The motion / echo node grid collapses to one device: ``--echo-groups`` and
``--motion-groups`` must be 1.
"""

from __future__ import annotations

import argparse
import json
import logging
import os
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .. import cfl as _cfl
from ..solver import PdhgSolver

ALGORITHMS = ("tvm", "tvme", "tvmw")


# ---------------------------------------------------------------------- flags
def build_parser(algorithm: str) -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(description=f"{algorithm.upper()} PDHG reconstruction (b200 backend, one GPU).")
    p.add_argument("--readout-fraction", "--frac", dest="frac", type=float, default=0.98)
    p.add_argument("--num-bins", "--num_bins", dest="num_bins", type=int, default=6)
    if algorithm == "tvm":
        p.add_argument("--lambda-motion", "--lamda", dest="lamda", type=float, default=1e-5)
        p.add_argument("--reduce-per-bin", "--reduce_per_bin", dest="reduce_per_bin", action="store_true")
    elif algorithm == "tvme":
        p.add_argument("--lambda-motion", "--lamda_m", dest="lamda_m", type=float, default=1e-5)
        p.add_argument("--lambda-echo", "--lamda_e", dest="lamda_e", type=float, default=1e-5)
    else:
        p.add_argument("--lambda-motion", "--lambda1", dest="lambda1", type=float, default=1e-5)
        p.add_argument("--lambda-echo-wavelet", "--lambda2", dest="lambda2", type=float, default=1e-5)
        p.add_argument("--lambda-spatial-wavelet", "--lambda3", dest="lambda3", type=float, default=1e-5)
    p.add_argument("--max-iter", "--max_iter", dest="max_iter", type=int, default=300)
    p.add_argument("--tol", type=float, default=1e-3)
    if algorithm != "tvmw":
        p.add_argument("--acceleration", "--acc", dest="acc", type=int, default=1)
    p.add_argument("--fov-scale", "--fov_scale", dest="fov_scale", type=float, nargs=3, default=[1.0, 1.0, 1.0])
    p.add_argument("--crop-to-original", "--crop_to_orig", dest="crop_to_orig", action="store_true")
    p.add_argument("--echo-groups", "--echo_groups", dest="echo_groups", type=int, default=1)
    p.add_argument("--motion-groups", "--motion_groups", dest="motion_groups", type=int, default=1)
    p.add_argument("--l2-coupling", "--l2_coupling", dest="l2_coupling", action="store_true")
    p.add_argument("--show-progress", "--show_pbar", dest="show_pbar", action="store_true")
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--multi-gpu", "--multi_gpu", dest="multi_gpu", action="store_true")
    p.add_argument("--fp16-communication", "--use_fp16_comm", dest="use_fp16_comm", action="store_true")
    p.add_argument("--nufft-backend", choices=("sigpy", "b200"), default="b200")
    p.add_argument("--warm-start", choices=("none", "learned"), default="none",
                   help="initial PDHG iterate: zeros (reference) or the learned network's prediction")
    p.add_argument("--no-cuda-graph", dest="cuda_graph", action="store_false")
    p.add_argument("--step-rule", choices=("reference", "power"), default="reference",
                   help="PDHG steps: the reference's sigma = tau = 1/6, or block-diagonal steps set by an FP64 "
                        "power-iteration estimate of the data operator norm")
    p.add_argument("--prepared-dir", type=str, default=None)
    p.add_argument("--output-dir", type=str, default=".")
    p.add_argument("--verbose", action="store_true")
    p.add_argument("input_dir", type=str)
    p.add_argument("img_file", type=str)
    return p


# ---------------------------------------------------------------------- preparation
@dataclass
class Prepared:
    ksp: np.ndarray          # (E, C, TR_sel, RO) complex64, normalised
    coord: np.ndarray        # (TR_sel, RO, 3) float32 zyx grid units
    dcf: np.ndarray          # (TR_sel, RO) float32
    resp: np.ndarray         # (TR_sel,) float
    mps: np.ndarray          # (C, Z, Y, X) complex64, normalised
    bin_edges: np.ndarray    # (B + 1,)
    img_shape: tuple
    orig_img_shape: tuple
    meta: dict = field(default_factory=dict)


def _read_triplet(path: str) -> list:
    with open(path, "r", encoding="utf-8") as fh:
        return fh.readline().strip().split(":")


def prepare(args, algorithm: str) -> Prepared:
    """Load and prepare one single-rank problem exactly as the reference's main does."""
    if args.echo_groups != 1 or args.motion_groups != 1:
        raise ValueError("the b200 backend runs the whole motion x echo grid on one device: "
                         "--echo-groups and --motion-groups must be 1")
    inp = args.input_dir
    prepared_dir = args.prepared_dir or inp
    img_shape = [int(v) for v in _read_triplet(os.path.join(inp, "imageDim.txt"))[::-1]]
    voxel = [float(v) for v in _read_triplet(os.path.join(inp, "voxelSize.txt"))[::-1]]
    orig_img_shape = list(img_shape)
    coord_full = np.squeeze(_cfl.read(os.path.join(inp, "ktraj"))).real[..., ::-1].astype(np.float32)
    dcf_full = np.squeeze(_cfl.read(os.path.join(inp, "dens"))).real.astype(np.float32)
    resp_full = np.squeeze(_cfl.read(os.path.join(prepared_dir, "resp"))).real
    num_tr_total = int(resp_full.size)
    if algorithm in ("tvm", "tvme"):
        tr_keep = np.arange(num_tr_total, dtype=np.int64)
        lo, hi = np.percentile(resp_full, 2), np.percentile(resp_full, 98)
        tr_keep = tr_keep[(resp_full > lo) & (resp_full < hi)]
        tr_keep = tr_keep[: int(num_tr_total / max(int(args.acc), 1))]
    else:
        tr_keep = np.arange(num_tr_total, dtype=np.int64)
    num_ro = int(args.frac * coord_full.shape[-2])
    coord = np.array(coord_full[tr_keep, :num_ro], dtype=np.float32)
    dcf = np.array(dcf_full[tr_keep, :num_ro], dtype=np.float32)
    resp = resp_full[tr_keep]
    while coord.max() > 1000:
        num_ro -= 1
        coord = coord[:, :num_ro]
        dcf = dcf[:, :num_ro]
    for d in range(coord.shape[-1]):
        coord[..., d] *= voxel[d] * img_shape[d]
    fov = np.asarray(args.fov_scale, dtype=float)
    if not np.allclose(fov, 1.0):
        if np.any(fov < 1.0):
            raise ValueError("FoV scale factors must be >= 1.0 for all axes (z y x).")
        coord = coord.copy()
        coord[..., 0] *= fov[-3]
        coord[..., 1] *= fov[-2]
        coord[..., 2] *= fov[-1]
        img_shape = [int(img_shape[-3] * fov[-3]), int(img_shape[-2] * fov[-2]), int(img_shape[-1] * fov[-1])]
    if algorithm in ("tvm", "tvme"):
        m = float(np.max(dcf))
        if m > 0:
            dcf /= np.float32(m)
    edges = np.percentile(resp, np.linspace(0, 100, args.num_bins + 1))
    mask = np.zeros(resp.shape, dtype=bool)
    for b in range(args.num_bins):
        mask |= (resp >= edges[b]) & (resp < edges[b + 1])
    idx = np.nonzero(mask)[0].astype(np.int64)
    coord, dcf, resp = coord[idx], dcf[idx], resp[idx]
    E_total = _cfl.kspace_layout(_cfl.read_header(os.path.join(inp, "ksp")))[0]
    ksp = _cfl.read_kspace(os.path.join(inp, "ksp"), 0, E_total, num_ro, tr_keep[idx])
    mps = _cfl.read_maps(os.path.join(prepared_dir, "mps"))
    if tuple(mps.shape[-3:]) != tuple(img_shape):
        raise ValueError(f"MPS grid {tuple(mps.shape[-3:])} does not match the requested reconstruction grid "
                         f"{tuple(img_shape)}. Prepare sensitivity maps with the same FoV scale.")
    kmax = float(np.max(np.abs(ksp))) if ksp.size else 0.0
    if kmax > 0:
        ksp /= np.float32(kmax)
    sos = np.sqrt(np.sum(np.abs(mps) ** 2, axis=0, dtype=np.float32))
    if algorithm == "tvme":
        sos = np.maximum(sos, np.float32(1e-12))
    else:
        sos[sos == 0] = np.float32(1.0)
    mps = (mps / sos[None]).astype(np.complex64)
    if algorithm in ("tvm", "tvmw"):
        m = float(np.max(dcf)) if dcf.size else 0.0
        if m > 0:
            dcf /= np.float32(m)
    return Prepared(ksp=ksp, coord=coord, dcf=dcf, resp=resp, mps=mps, bin_edges=edges,
                    img_shape=tuple(img_shape), orig_img_shape=tuple(orig_img_shape),
                    meta={"num_ro": num_ro, "voxel_size": voxel, "fov_scale": fov.tolist(), "E_total": E_total,
                          "prepared_dir": prepared_dir})


# ---------------------------------------------------------------------- reconstructors
class _Reconstructor:
    """Shared constructor logic of the reference reconstructors on one device."""

    algorithm = "tvme"

    def __init__(self, ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling=False, *, sigma=0.01, tau=0.01,
                 max_iter=300, tol=1e-3, margin=10, device=0, E_total=None, e0=None, e1=None, echo_left_peer=None,
                 echo_right_peer=None, B_total=None, b0=None, b1=None, motion_left_peer=None,
                 motion_right_peer=None, bin_edges=None, world_comm=None, group_comm=None, leader_comm=None,
                 nccl_group=None, dist_grid=None, tagger=None, show_pbar=True, nufft_backend="b200",
                 lam=None, warm_start=None, use_graph=True, step_rule="reference"):
        if str(nufft_backend).lower() != "b200":
            raise ValueError("these reconstructors run the b200 backend; the SigPy path is the reference's own code")
        self.E = int(ksp.shape[0])
        self.B = int(B_local)
        B_total = self.B if B_total is None else int(B_total)
        if B_total != self.B or (E_total is not None and int(E_total) != self.E):
            raise ValueError("one device holds every motion bin and echo (B_total == B_local, E_total == E)")
        for peer in (echo_left_peer, echo_right_peer, motion_left_peer, motion_right_peer):
            if peer not in (None, -2):   # MPI.PROC_NULL
                raise ValueError("halo peers are not used: the b200 backend runs on one device")
        if bin_edges is None:
            bins = np.percentile(resp, np.linspace(0 + margin, 100 - margin, B_total + 1))
        else:
            bins = np.asarray(bin_edges)
            if bins.ndim != 1 or bins.size != B_total + 1:
                raise ValueError(f"bin_edges must have shape ({B_total + 1},), got {bins.shape}")
        coords, dcfs, ksps = [], [], []
        for gb in range(B_total):
            idx = (resp >= bins[gb]) & (resp < bins[gb + 1])
            coords.append(np.asarray(coord)[idx])
            dcfs.append(np.asarray(dcf)[idx])
            ksps.append(np.asarray(ksp)[:, :, idx])
        self.img_shape = tuple(int(v) for v in np.asarray(mps).shape[-3:])
        self.max_iter, self.tol = int(max_iter), float(tol)
        self.show_pbar = show_pbar
        self.warm_start = warm_start
        self.solver = PdhgSolver(self.algorithm, self.img_shape, coords, dcfs, mps, ksps, device=device,
                                 l2_coupling=l2_coupling, sigma=sigma, tau=tau, use_graph=use_graph,
                                 step_rule=step_rule, **(lam or {}))
        self.result = None

    def run(self):
        """Run PDHG to ``tol`` / ``max_iter``; returns u_bar (B, E, Z, Y, X) on the GPU."""
        t0 = time.perf_counter()
        if self.warm_start is not None:
            from ..warmstart import warm_solve
            self.result = warm_solve(self.solver, None, max_iter=self.max_iter, tol=self.tol, model=self.warm_start)
        else:
            self.result = self.solver.run(max_iter=self.max_iter, tol=self.tol)
        logging.info("[PDHG iterations only] %.2f s (device), %d iterations, %.2f s wall",
                     self.result.seconds, self.result.iterations, time.perf_counter() - t0)
        return self.result.image


class TvmReconstructor(_Reconstructor):
    algorithm = "tvm"

    def __init__(self, ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling=False, lamda=1e-5, **kw):
        kw.pop("reduce_per_bin", None)
        super().__init__(ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling, lam={"lam_m": lamda}, **kw)


class TvmeReconstructor(_Reconstructor):
    algorithm = "tvme"

    def __init__(self, ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling=False, lamda_m=1e-5,
                 lamda_e=1e-5, **kw):
        super().__init__(ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling,
                         lam={"lam_m": lamda_m, "lam_e": lamda_e}, **kw)


class TvmwReconstructor(_Reconstructor):
    algorithm = "tvmw"

    def __init__(self, ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling=False, lambda1=1e-5,
                 lambda2=1e-5, lambda3=1e-5, **kw):
        super().__init__(ksp, coord, dcf, mps, resp, dual_q, B_local, l2_coupling,
                         lam={"lam_m": lambda1, "lam_w1": lambda2, "lam_w2": lambda3}, **kw)


RECONSTRUCTORS = {"tvm": TvmReconstructor, "tvme": TvmeReconstructor, "tvmw": TvmwReconstructor}


def _lambdas(args, algorithm):
    if algorithm == "tvm":
        return {"lamda": args.lamda}
    if algorithm == "tvme":
        return {"lamda_m": args.lamda_m, "lamda_e": args.lamda_e}
    return {"lambda1": args.lambda1, "lambda2": args.lambda2, "lambda3": args.lambda3}


def _manifest_parameters(args, algorithm, E_total):
    par = {"readout_fraction": args.frac, "num_bins": args.num_bins, "num_echoes": E_total,
           "max_iter": args.max_iter, "tol": args.tol, "fov_scale_zyx": list(args.fov_scale),
           "crop_to_original": args.crop_to_orig, "l2_coupling": args.l2_coupling}
    if algorithm == "tvm":
        par.update(lambda_motion=args.lamda, acceleration=args.acc, reduce_per_bin=args.reduce_per_bin)
    elif algorithm == "tvme":
        par.update(lambda_motion=args.lamda_m, lambda_echo=args.lamda_e, acceleration=args.acc)
    else:
        par.update(lambda_motion=args.lambda1, lambda_echo_wavelet=args.lambda2, lambda_spatial_wavelet=args.lambda3)
    return par


def center_crop_zyx(arr, out_shape_zyx):
    Nz0, Ny0, Nx0 = out_shape_zyx
    Nz, Ny, Nx = arr.shape[-3:]
    if Nz0 > Nz or Ny0 > Ny or Nx0 > Nx:
        raise ValueError(f"Requested crop {out_shape_zyx} larger than input {(Nz, Ny, Nx)}")
    z0, y0, x0 = (Nz - Nz0) // 2, (Ny - Ny0) // 2, (Nx - Nx0) // 2
    return arr[..., z0:z0 + Nz0, y0:y0 + Ny0, x0:x0 + Nx0]


def main_for(algorithm: str, argv=None) -> int:
    start = time.perf_counter()
    args = build_parser(algorithm).parse_args(argv)
    if args.verbose:
        logging.basicConfig(level=logging.DEBUG)
    if args.nufft_backend != "b200":
        raise SystemExit("--nufft-backend sigpy runs the reference's own reconstructor (toporecon); "
                         "this entry point implements --nufft-backend b200")
    prep = prepare(args, algorithm)
    warm = None
    if args.warm_start == "learned":
        from ..warmstart import load_model
        warm = load_model()
    rec = RECONSTRUCTORS[algorithm](prep.ksp, prep.coord, prep.dcf, prep.mps, prep.resp, None, args.num_bins,
                                    args.l2_coupling, sigma=1 / 6, tau=1 / 6, max_iter=args.max_iter, tol=args.tol,
                                    margin=0, device=args.device, E_total=prep.meta["E_total"], e0=0,
                                    e1=prep.meta["E_total"], B_total=args.num_bins, b0=0, b1=args.num_bins,
                                    bin_edges=prep.bin_edges, show_pbar=args.show_pbar, nufft_backend="b200",
                                    warm_start=warm, use_graph=args.cuda_graph, step_rule=args.step_rule,
                                    **_lambdas(args, algorithm))
    image = rec.run().cpu().numpy()
    B, E = image.shape[:2]
    Z, Y, X = image.shape[-3:]
    out = np.zeros((B, 1, 1, E, 1, 1, Z, Y, X), dtype=np.complex64)
    out[:, 0, 0, :, 0, 0] = image
    if args.crop_to_orig and not np.allclose(np.asarray(args.fov_scale), 1.0):
        out = center_crop_zyx(out, prep.orig_img_shape)
    os.makedirs(args.output_dir, exist_ok=True)
    E_total = prep.meta["E_total"]
    stem = f"{args.img_file}_e0-{E_total - 1}_m0-{args.num_bins - 1}"
    _cfl.write(os.path.join(args.output_dir, stem), out)
    res = rec.result
    manifest = {
        "format_version": 1, "algorithm": algorithm, "nufft_backend": "b200",
        "input_directory": os.path.abspath(args.input_dir),
        "prepared_directory": os.path.abspath(prep.meta["prepared_dir"]),
        "output_stem": args.img_file, "output_pattern": f"{args.img_file}_e{{e0}}-{{e1}}_m{{b0}}-{{b1}}",
        "parameters": _manifest_parameters(args, algorithm, E_total),
        "distributed": {"world_size": 1, "num_nodes": 1, "motion_groups": 1, "echo_groups": 1,
                        "fp16_communication": args.use_fp16_comm},
        "normalization": {"kspace": "global_max_magnitude", "mps": "coil_root_sum_of_squares",
                          "density": "maximum" if algorithm == "tvme" else "global_maximum_after_motion_sharding"},
        "b200": {"iterations": res.iterations, "final_tol": res.tols[-1] if res.tols else None,
                 "pdhg_seconds": res.seconds, "sigma": res.sigma, "tau": res.tau, "sigma_data": res.sigma_data,
                 "step_rule": res.step_rule, "data_norm": res.data_norm, "warm_start": args.warm_start,
                 "cuda_graph": bool(args.cuda_graph), "main_seconds": time.perf_counter() - start},
    }
    with open(os.path.join(args.output_dir, "run_manifest.json"), "w", encoding="utf-8") as fh:
        json.dump(manifest, fh, indent=2, sort_keys=True)
        fh.write("\n")
    rec.solver.close()
    return 0
