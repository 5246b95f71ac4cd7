#!/usr/bin/env python3
"""Benchmark of the b200 PDHG backend (toporecon TVME / TVM / TVMW).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config tvme-256] [--impl b200|reference]

Workload (default ``tvme-256``): TVME at 256 x 256 x 128, 16 coils, 6 echoes,
6 motion bins, 4096 cones x 800 readout points, lambda 1e-5, tol 1e-3, max 1000
iterations (a cap the solve does not reach), seeded synthetic phantom (the reference's liver dataset is not
available).  A "step" is one PDHG iteration over the whole batch (every bin,
echo and coil).  W warm-up steps, then K steps timed with CUDA events on the
solver's stream; then a full plain (zero-start) solve to tolerance and, when a
trained network is present, a warm-started solve, each timed with CUDA events.
Both solves use ``--step-rule`` (default ``power``: block-diagonal PDHG steps
from the FP64 power-iteration estimate of the data operator norm, whose device
time is part of every solve's time; ``reference``: sigma = tau = 1/6).

The JSON line's ``value`` is the time-to-tolerance in seconds: the
warm-started solve when a trained network exists, it reached the tolerance and
its result is within 1e-3 relative L2 of the plain result, else the plain
solve (``value_source`` says which); inputs are resident in HBM when timing
starts.  ``tol_reached_plain`` says whether the plain solve met ``--tol``
before ``max_iter``.  ``oracle_check`` gives the relative L2 errors of the
b200 NUFFT (against the FP64 direct NUDFT and the KB restatement) and of a
short PDHG run with the same steps (against the FP64 PDHG oracle) on a 32^3
crop of the workload; it runs after every timed region.
``e2e`` is the same solve through the public API from pinned host buffers
(plan creation, H2D of k-space and maps, sort, solve, D2H of the image).
``roofline`` reports the dominant NUFFT kernel (CUDA-event time of one launch
on the full workload) against the measured HBM copy bandwidth.
``cpu_baseline`` times the CPU oracle port (C/OpenMP KB loops + scipy.fft) on
a bounded sample (one bin-echo-coil forward + adjoint NUFFT at full size plus
one PDHG elementwise slice) scaled to the solve.

Multi-GPU (torchrun): the motion bins of the same problem are split over the
ranks by sample count, with the one-bin halos of u_bar and p_m and the two
stopping sums passed over NCCL each iteration (``parallel.py``); strong
scaling, times are the max over ranks.
Inputs exceed L2 (126 MB): every k-space column block and grid is larger.
"""

from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from dataclasses import replace
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))
PKG = "multinodemri-miccai26_b200"
METRIC = "TVME time-to-tol 1e-3 (s) on 1 B200, warm-start vs plain PDHG; NUFFT GB/s"
FALLBACK_HBM_GBS = 6650.0
WARM_MATCH = 1e-3      # warm-started result must match the plain result to this relative L2

# DRAM bytes (read + write) of one launch of each NUFFT stage, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on one bin of this trajectory
# and grid with 16 k-space columns (profiles/nufft_pdhg_kernels_256x256x128_16col.md);
# the grid-sized traffic scales with the column count, so roofline.traffic for the
# 96-column bench workload is these figures x ncol / 16.
NCU_TRAFFIC_16COL = {
    "workload": "tvme-256", "columns": 16,
    "fwd_x": 1.962e9, "fwd_y": 2.973e9, "fwd_z": 3.019e9, "interp": 1.304e9,
    "spread": 2.296e9, "adj_z": 3.326e9, "adj_y": 2.982e9, "adj_x": 2.012e9,
}

# Iterations to --tol of plain PDHG with the reference's steps (sigma = tau =
# 1/6) on each seeded workload, measured with the b200 arm on the same seeded
# problem (TVME-256: `bench.py --step-rule reference --max-iter 2000`, tol
# 0.000999 at iteration 510); None: the configuration's max_iter (the rule is not
# met before it).  The CPU reference arm cannot run a full solve within minutes
# and extrapolates its per-iteration time with these.
ITERS_TO_TOL = {"tvme-256": 510, "tvme-256-dirichlet": None, "tvme-128": None, "tvmw-160": None, "tvm-64": 100}


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[1])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--config", default="tvme-256")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the workload (debug runs only)")
    ap.add_argument("--max-iter", type=int, default=None)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--jsense", action="store_true",
                    help="time JSENSE coil-map estimation on the workload's first echo instead of PDHG")
    ap.add_argument("--sharded", action="store_true",
                    help="use the bin-sharded multi-GPU path even on one GPU (exercises its code on one device)")
    ap.add_argument("--step-rule", choices=("power", "reference"), default="power",
                    help="PDHG steps of the timed solves: block-diagonal steps from the FP64 power-iteration "
                         "norm estimate (default), or the reference's sigma = tau = 1/6")
    ap.add_argument("--no-warm", action="store_true", help="skip the warm-started solve")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the FP64-oracle error report on the small crop of the workload")
    return ap.parse_args(argv)


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


def get_config(args):
    syn = importlib.import_module(f"{PKG}.synthetic")
    cfg = syn.CONFIGS[args.config]
    if args.scale != 1.0:
        cfg = syn.scaled(cfg, args.scale)
    if args.max_iter:
        cfg = replace(cfg, max_iter=args.max_iter)
    return cfg


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "of measured"
    return FALLBACK_HBM_GBS, "of fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")
        sm = [num(r[1]) for r in rows]
        pw = [num(r[3]) for r in rows]
        smax = max(num(r[2]) for r in rows)
        load = [s for s, p in zip(sm, pw) if p > 250] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": smax, "reasons": reasons, "samples": len(rows)}


def dist_setup(force: bool = False):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 or force:
        import datetime
        import torch.distributed as dist
        if force and "MASTER_ADDR" not in os.environ:
            os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": "29517", "RANK": "0", "WORLD_SIZE": "1"})
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x: float, world: int, device) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------- CPU baseline
def cpu_sample(cfg, ds_coord_bins, n_pairs: int = 1):
    """Time the oracle port on a bounded sample: n_pairs full-size (b, e, c)
    forward + adjoint NUFFTs and one elementwise TVME slice; returns seconds
    per PDHG iteration extrapolated to the whole batch, and the threads used."""
    from oracle import cgrid
    cgrid.build()
    rng = np.random.default_rng(123)
    shape = tuple(cfg.img_shape)
    k = ds_coord_bins[0].reshape(-1, 3)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    t0 = time.perf_counter()
    for _ in range(n_pairs):
        y = cgrid.nufft(x, k)
        cgrid.nufft_adjoint(y, k, shape)
    t_pair = (time.perf_counter() - t0) / n_pairs
    # elementwise: the oracle's TVME dual + primal on one (bin, echo-pair) slice
    from oracle import pdhg as op
    sl = (1, min(2, cfg.n_echoes)) + shape
    u = (rng.standard_normal(sl) + 1j * rng.standard_normal(sl)).astype(np.complex64)
    t0 = time.perf_counter()
    d = op.dxf(u) + op.dyf(u) + op.dzf(u)
    pm = u / np.maximum(1.0, np.abs(u) / 1e-5)
    dv = op.dxb(d) + op.dyb(d) + op.dzb(d)
    u2 = u - (1 / 6) * (dv + pm)
    _ = 2 * u2 - u
    t_elem = (time.perf_counter() - t0) * (cfg.n_bins * cfg.n_echoes) / (sl[0] * sl[1])
    per_iter = t_pair * cfg.n_bins * cfg.n_echoes * cfg.n_coils + t_elem
    return per_iter, cgrid.threads(), t_pair, t_elem


def oracle_check(cfg, step_rule: str, device: int, n_iter: int = 8) -> dict:
    """Relative L2 errors of the b200 path against the FP64 oracle on a 32^3
    crop of the workload (same algorithm, coupling, lambda, step rule,
    synthetic model; 4 coils, 2 echoes, 2 bins of 128 cones x 160 readout):
    the NUFFT against the FP64 direct NUDFT and the KB restatement, and
    ``n_iter`` PDHG iterations against the FP64 PDHG oracle with the same steps."""
    import torch
    from dataclasses import replace
    from oracle import cgrid
    from oracle import nufft as onf
    from oracle import pdhg as op
    syn = importlib.import_module(f"{PKG}.synthetic")
    solver_mod = importlib.import_module(f"{PKG}.solver")
    nb = importlib.import_module(f"{PKG}.nufft_backend")
    small = replace(cfg, name=cfg.name + "-crop32", img_shape=(32, 32, 32), n_coils=4,
                    n_echoes=min(2, cfg.n_echoes), n_bins=2, n_interleaves=128, n_readout=160,
                    binning="amplitude")
    ds = syn.make_geometry(small)
    syn.simulate_kspace(ds, lambda imgs, k: cgrid.nufft(imgs, k))
    coords = [ds.coord[ds.bin_indices(b)].reshape(-1, 3) for b in range(small.n_bins)]
    dcfs = [ds.dcf[ds.bin_indices(b)].reshape(-1) for b in range(small.n_bins)]
    ksps = [ds.ksp[:, :, ds.bin_indices(b)].reshape(small.n_echoes, small.n_coils, -1) for b in range(small.n_bins)]
    # NUFFT of one image at bin 0's samples: FP64 direct NUDFT and the KB restatement
    be = nb.B200NufftBackend(small.img_shape, [coords[0]], device)
    x = ds.truth[0, 0]
    y = be.forward(x, 0)
    be.close()
    nudft = onf.nudft(x.astype(np.complex128), coords[0])
    kb = onf.nufft(x, coords[0])
    lam = small.lam
    s = solver_mod.PdhgSolver(small.algorithm, small.img_shape, coords, dcfs, ds.mps, ksps, device=device,
                              l2_coupling=small.l2_coupling, lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam,
                              step_rule=step_rule, power_iters=40)
    r = s.run(max_iter=n_iter, tol=0.0)
    img = r.image.cpu().numpy()
    s.close()
    pb = op.Problem(op.OracleNufft(small.img_shape, coords), [k.astype(np.complex128) for k in ksps], dcfs, ds.mps)
    ref = op.run(small.algorithm, pb, max_iter=n_iter, tol=0.0, sigma=r.sigma, tau=r.tau, sigma_data=r.sigma_data,
                 lam_m=lam, lam_e=lam, lam1=lam, lam2=lam, lam3=lam, l2_coupling=small.l2_coupling)
    torch.cuda.synchronize()
    return {"crop": list(small.img_shape), "coils": small.n_coils, "echoes": small.n_echoes, "bins": small.n_bins,
            "pdhg_iterations": n_iter, "step_rule": step_rule,
            "rel_l2_pdhg_vs_fp64_pdhg": onf.rel_l2(img, ref.image),
            "rel_l2_nufft_vs_fp64_nudft": onf.rel_l2(y, nudft),
            "rel_l2_nufft_vs_kb_restatement": onf.rel_l2(y, kb),
            "kb_restatement_vs_fp64_nudft": onf.rel_l2(kb, nudft)}


def bin_coords(ds):
    return [ds.coord[ds.bin_indices(b)] for b in range(ds.cfg.n_bins)]


# --------------------------------------------------------------------------- b200 arm
def run_b200(args):
    import torch
    world, rank, local = dist_setup(force=args.sharded)
    torch.cuda.set_device(local)
    if world > 1 or args.sharded:
        run_b200_sharded(args, world, rank, local)
        import torch.distributed as dist
        dist.destroy_process_group()
        return
    device = torch.device("cuda", local)
    syn = importlib.import_module(f"{PKG}.synthetic")
    solver_mod = importlib.import_module(f"{PKG}.solver")
    cfg = get_config(args)
    t0 = time.perf_counter()
    ds = syn.make_geometry(cfg)
    log(f"geometry {time.perf_counter() - t0:.1f}s")
    t0 = time.perf_counter()
    syn.simulate_kspace_b200(ds, local)
    log(f"k-space simulated on the GPU in {time.perf_counter() - t0:.1f}s")
    coords, dcfs, ksps = bin_coords(ds), ds.bin_dcf(), ds.bin_ksp()
    lam = cfg.lam
    t0 = time.perf_counter()
    solver = solver_mod.PdhgSolver(cfg.algorithm, cfg.img_shape, coords, dcfs, ds.mps, ksps,
                                   l2_coupling=cfg.l2_coupling, lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam,
                                   use_graph=not args.no_graph, device=local)
    log(f"solver set up in {time.perf_counter() - t0:.1f}s")
    st = solver.stream
    E, C, B = solver.E, solver.C, solver.B
    ncol = E * C
    # per bin: x, y, z passes + interpolation; gridding + split-tile reduction + z, y, x passes;
    # per iteration: TV duals, primal, tolerance reduction
    launches_per_iter = B * (4 + math.ceil(ncol / 128) + 1 + 3) + 3
    if cfg.algorithm == "tvmw":
        launches_per_iter += 6 * max(1, solver.backend.wavelet_levels)

    clocks = ClockSampler(local)
    # ---- warm-up and K timed steps (one PDHG iteration each)
    solver.reset()
    solver.iterate(max(3, args.warmup), tol=0.0)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(st)
    solver.iterate(args.steps, tol=0.0)
    ev1.record(st)
    ev1.synchronize()
    torch.cuda.synchronize()
    ms_step = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world, device)

    # ---- plain solve to tolerance (the power rule's norm estimate is part of its time)
    if args.step_rule == "power":
        solver.set_power_steps()
        log(f"power rule: ||W^1/2 A|| = {solver.data_norm:.6g} ({solver.setup_seconds:.3f}s), sigma {solver.sigma:.4g}, "
            f"tau {solver.tau:.4g}, sigma_data {solver.sigma_data:.4g}")
    r_plain = solver.run(max_iter=cfg.max_iter, tol=cfg.tol)
    plain_img = r_plain.image.clone()
    t_plain = max_over_ranks(r_plain.seconds + r_plain.setup_seconds, world, device)
    log(f"plain: {r_plain.iterations} iterations, {t_plain:.3f}s (tol {r_plain.tols[-1]:.3g})")

    # ---- warm-started solve (learned initial iterate), when a trained network exists
    warm = None
    try:
        if args.no_warm or cfg.algorithm != "tvme":
            raise FileNotFoundError("not requested (the network is trained for TVME)")
        ws = importlib.import_module(f"{PKG}.warmstart")
        warm = ws.warm_solve(solver, cfg, max_iter=cfg.max_iter, tol=cfg.tol)
    except (ImportError, FileNotFoundError, AttributeError) as exc:
        log(f"warm start unavailable: {exc}")
    clk = clocks.stop()

    # ---- per-stage profile of bin 0 (roofline)
    prof = solver.backend.profile(0, reps=3)
    hbm, peak_src = peaks()
    used = solver.backend.pipeline(prof)          # the stages a solve runs (fused y / z passes or not)
    dom_name = max(used, key=lambda k: prof[k]["ms"])
    dom = prof[dom_name]
    nufft_ms = sum(prof[k]["ms"] for k in used)
    traffic, traffic_src = None, None
    if cfg.name == NCU_TRAFFIC_16COL["workload"] and dom_name in NCU_TRAFFIC_16COL:
        traffic = round(NCU_TRAFFIC_16COL[dom_name] * (E * C) / NCU_TRAFFIC_16COL["columns"])
        traffic_src = f"ncu DRAM bytes at 16 columns x {E * C}/16"
    nufft_bytes = sum(prof[k]["bytes"] for k in used)

    # ---- FP64 oracle agreement and warm/plain agreement
    rel_warm = None
    if warm is not None:
        a = warm.image.reshape(-1)
        rel_warm = float(torch.linalg.vector_norm(a - plain_img.reshape(-1)) /
                         torch.linalg.vector_norm(plain_img.reshape(-1)))

    # the warm-started time counts only when its answer is the plain PDHG answer
    # (relative L2 within WARM_MATCH) and it reached the tolerance; otherwise the plain time is the value
    t_warm = None if warm is None else warm.seconds + warm.setup_seconds
    use_warm = (warm is not None and rel_warm is not None and rel_warm <= WARM_MATCH
                and warm.tols and warm.tols[-1] < cfg.tol)
    value = max_over_ranks(t_warm if use_warm else t_plain, world, device)

    # ---- e2e through the public API from pinned host buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        ksp_h = [pin(k) for k in ksps]
        mps_h = pin(ds.mps)
        h2d = sum(k.numel() * 8 for k in ksp_h) + mps_h.numel() * 8 + sum(c.size * 4 for c in coords) + \
            sum(d.size * 4 for d in dcfs)
        solver.close()
        del solver
        torch.cuda.empty_cache()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2 = solver_mod.PdhgSolver(cfg.algorithm, cfg.img_shape, coords, dcfs, mps_h, ksp_h,
                                   l2_coupling=cfg.l2_coupling, lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam,
                                   use_graph=not args.no_graph, device=local, step_rule=args.step_rule)
        if use_warm:
            r2 = ws.warm_solve(s2, cfg, max_iter=cfg.max_iter, tol=cfg.tol)
        else:
            r2 = s2.run(max_iter=cfg.max_iter, tol=cfg.tol)
        out_h = torch.empty(r2.image.shape, dtype=torch.complex64, pin_memory=True)
        out_h.copy_(r2.image, non_blocking=True)
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(time.perf_counter() - t0, world, device)
        e2e = {"value": round(t_e2e, 4), "unit": "s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(out_h.numel() * 8)}
        s2.close()

    # ---- FP64-oracle error on a small crop of the workload (checker, outside every timed region)
    check = None
    if rank == 0 and world == 1 and not args.no_oracle_check:
        check = oracle_check(cfg, args.step_rule, local)
        log(f"oracle check: {check}")

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        per_iter, threads, t_pair, t_elem = cpu_sample(cfg, coords)
        cpu = {"value": round(per_iter * r_plain.iterations, 2), "unit": "s", "cores": threads, "kind": "port",
               "sample": f"one full-size bin-echo-coil forward+adjoint NUFFT ({t_pair:.2f}s) x {B * E * C} "
                         f"+ elementwise slice ({t_elem:.2f}s/iter), times {r_plain.iterations} plain iterations"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": round(value, 4),
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(3, args.warmup),
            "ms_per_step": round(ms_step, 3),
            "higher_is_better": False,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "c64",
            "data": "synthetic",
            "config": {"workload": cfg.name, "algorithm": cfg.algorithm, "img_shape_zyx": list(cfg.img_shape),
                       "coils": C, "echoes": E, "bins": B, "cones": cfg.n_interleaves, "readout": cfg.n_readout,
                       "tol": cfg.tol, "max_iter": cfg.max_iter, "l2_flush": "inputs larger than L2",
                       "step_rule": args.step_rule,
                       "parallelism": "replicas" if world > 1 else "single-gpu"},
            "value_source": ("warm-started PDHG" if use_warm else "plain PDHG") + f", {args.step_rule} step rule",
            "pdhg_steps": {"sigma": r_plain.sigma, "tau": r_plain.tau, "sigma_data": r_plain.sigma_data,
                           "data_norm": r_plain.data_norm, "norm_estimate_s": round(r_plain.setup_seconds, 4)},
            "tol_reached_plain": bool(r_plain.tols and r_plain.tols[-1] < cfg.tol),
            "time_to_tol_plain_s": round(t_plain, 4),
            "iterations_plain": r_plain.iterations,
            "tol_trace_plain": [round(t, 6) for t in r_plain.tols[::max(1, len(r_plain.tols) // 12)]],
            "time_to_tol_warm_s": None if warm is None else round(t_warm, 4),
            "iterations_warm": None if warm is None else warm.iterations,
            "tol_reached_warm": None if warm is None else bool(warm.tols and warm.tols[-1] < cfg.tol),
            "warm_speedup": None if warm is None else round(t_plain / t_warm, 3),
            "rel_l2_warm_vs_plain": rel_warm,
            "oracle_check": check,
            "iterations_per_s": round(1000.0 / ms_step, 3),
            "nufft_gbs": round(nufft_bytes / (nufft_ms * 1e6), 1),
            "nufft_stages": {k: {"ms": round(v["ms"], 4), "gbs": round(v["gbs"], 1),
                                 "frac": round(v["gbs"] / hbm, 3)} for k, v in prof.items()},
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(dom["gbs"], 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(dom["gbs"] / hbm, 3), "peak_source": peak_src,
                         "traffic": traffic, "traffic_source": traffic_src, "algorithmic_bytes": dom["bytes"],
                         "launch_ms": round(dom["ms"], 4)},
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "gpu_launches": launches_per_iter * args.steps,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# --------------------------------------------------------------------------- b200 arm, several GPUs
def run_b200_sharded(args, world, rank, local):
    """N ranks, one GPU each: the motion bins of the one problem split by
    sample count (``parallel.partition_bins``), halos and the stopping sums over
    NCCL.  Strong scaling: the whole job is the same single problem."""
    import torch
    device = torch.device("cuda", local)
    syn = importlib.import_module(f"{PKG}.synthetic")
    solver_mod = importlib.import_module(f"{PKG}.solver")
    par = importlib.import_module(f"{PKG}.parallel")
    cfg = get_config(args)
    ds = syn.make_geometry(cfg)
    syn.simulate_kspace_b200(ds, local)
    coords, dcfs, ksps = bin_coords(ds), ds.bin_dcf(), ds.bin_ksp()
    counts = [int(np.prod(c.shape[:-1])) for c in coords]
    ranges = par.partition_bins(counts, world)
    a, e = ranges[rank]
    lam = cfg.lam
    comm = par.TorchHaloComm(ranges)

    def build(mps, ksp_list):
        if e <= a:
            return None, par.IdleEngine(device)
        sv = solver_mod.PdhgSolver(cfg.algorithm, cfg.img_shape, coords[a:e], dcfs[a:e], mps, ksp_list[a:e],
                                   l2_coupling=cfg.l2_coupling, lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam,
                                   device=local)
        return sv, par.B200ShardEngine(sv, a, len(counts))

    solver, eng = build(ds.mps, ksps)
    sh = par.ShardedPdhg(eng, comm, cfg.algorithm)
    clocks = ClockSampler(local)
    eng.reset(None)
    sh.iterate(max(3, args.warmup), 0.0, 1 / 6, 1 / 6)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    t = eng.timer()
    t.start()
    sh.iterate(args.steps, 0.0, 1 / 6, 1 / 6)
    ms_step = max_over_ranks(t.stop() * 1e3 / args.steps, world, device)
    res = sh.run(max_iter=cfg.max_iter, tol=cfg.tol)
    t_plain = max_over_ranks(res.seconds, world, device)
    clk = clocks.stop()
    e2e = None
    if not args.no_e2e:
        pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
        ksp_h = [pin(k) if a <= i < e else None for i, k in enumerate(ksps)]
        mps_h = pin(ds.mps)
        h2d = sum(k.numel() * 8 for k in ksp_h if k is not None) + mps_h.numel() * 8 + \
            sum(c.size * 4 for c in coords[a:e]) + sum(d.size * 4 for d in dcfs[a:e])
        if solver is not None:
            solver.close()
        del solver, eng, sh
        torch.cuda.empty_cache()
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s2, eng2 = build(mps_h, ksp_h)
        r2 = par.ShardedPdhg(eng2, comm, cfg.algorithm).run(max_iter=cfg.max_iter, tol=cfg.tol)
        d2h = 0
        if r2.image is not None:
            out_h = torch.empty(r2.image.shape, dtype=torch.complex64, pin_memory=True)
            out_h.copy_(r2.image, non_blocking=True)
            d2h = out_h.numel() * 8
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(time.perf_counter() - t0, world, device)
        e2e = {"value": round(t_e2e, 4), "unit": "s", "h2d_bytes_per_step": int(max_over_ranks(h2d, world, device)),
               "d2h_bytes_per_step": int(max_over_ranks(d2h, world, device))}
        if s2 is not None:
            s2.close()
    if rank == 0:
        E, C = cfg.n_echoes, cfg.n_coils
        line = {
            "metric": METRIC, "value": round(t_plain, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(ms_step, 3), "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
            "config": {"workload": cfg.name, "algorithm": cfg.algorithm, "img_shape_zyx": list(cfg.img_shape),
                       "coils": C, "echoes": E, "bins": cfg.n_bins, "cones": cfg.n_interleaves,
                       "readout": cfg.n_readout, "tol": cfg.tol, "max_iter": cfg.max_iter,
                       "l2_flush": "inputs larger than L2",
                       "parallelism": f"motion bins over {world} GPUs, NCCL halos",
                       "bins_per_rank": [int(y - x) for x, y in ranges]},
            "value_source": "plain PDHG",
            "time_to_tol_plain_s": round(t_plain, 4), "iterations_plain": res.iterations,
            "iterations_per_s": round(1000.0 / ms_step, 3),
            "clocks": clk, "e2e": e2e, "cpu_baseline": None,
            "gpu_launches": (max(e - a for a, e in ranges) * (8 + 1) + 3) * args.steps,
        }
        print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- reference arm
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = get_config(args)
    syn = importlib.import_module(f"{PKG}.synthetic")
    rng = np.random.default_rng(cfg.seed)
    coord = syn.cones_trajectory(cfg.img_shape, cfg.n_interleaves, cfg.n_readout, rng)
    nb = cfg.n_bins
    per_bin = coord[: max(1, cfg.n_interleaves // nb)]
    iters = ITERS_TO_TOL.get(cfg.name) or cfg.max_iter
    samples = []
    for i in range(max(0, args.warmup) + args.steps):
        t0 = time.perf_counter()
        per_iter, threads, t_pair, t_elem = cpu_sample(cfg, [per_bin])
        if i >= args.warmup:
            samples.append(per_iter)
    per_iter = statistics.mean(samples)
    value = per_iter * iters
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(per_iter * 1e3, 1), "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "c64", "data": "synthetic", "impl": "reference",
        "config": {"workload": cfg.name, "algorithm": cfg.algorithm, "img_shape_zyx": list(cfg.img_shape),
                   "coils": cfg.n_coils, "echoes": cfg.n_echoes, "bins": cfg.n_bins, "tol": cfg.tol},
        "iterations": iters,
        "cpu_baseline": {"value": round(value, 2), "unit": "s", "cores": threads, "kind": "port",
                         "sample": f"per step: one full-size bin-echo-coil NUFFT forward+adjoint x "
                                   f"{cfg.n_bins * cfg.n_echoes * cfg.n_coils} + elementwise slice; "
                                   f"x {iters} iterations"},
        "e2e": {"value": round(value, 2), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- JSENSE leg
def run_jsense(args):
    """JSENSE (SigPy application defaults: kernel 16, calibration 24, 10 x 10 CG
    iterations) on the workload's first echo: the b200 version timed whole (wall
    clock around a synchronised call), the CPU restatement (C/OpenMP KB loops,
    multi-threaded FFTs) timed on one outer iteration with two CG steps per
    sub-problem and scaled by NUFFT-pair count."""
    import torch
    syn = importlib.import_module(f"{PKG}.synthetic")
    js = importlib.import_module(f"{PKG}.jsense")
    cfg = get_config(args)
    ds = syn.make_geometry(cfg)
    syn.simulate_kspace_b200(ds, 0)
    coord = ds.coord.reshape(-1, 3)
    y0 = ds.ksp[0].reshape(cfg.n_coils, -1)
    keep = np.all(np.abs(coord) < 12.0, axis=-1)
    times = []
    for i in range(max(1, args.warmup) + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        maps = js.estimate_sensitivity_maps(ds.ksp[:1], ds.coord, ds.dcf, image_shape_zyx=cfg.img_shape)
        torch.cuda.synchronize()
        if i >= max(1, args.warmup):
            times.append(time.perf_counter() - t0)
    t_gpu = statistics.median(times)
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import jsense as oj
        from oracle import cgrid
        t0 = time.perf_counter()
        cgrid.build()
        oj.jsense(y0, coord, ds.dcf.reshape(-1), max_iter=1, inner=2, nufft=cgrid.nufft,
                  nufft_adjoint=cgrid.nufft_adjoint)
        t_cpu_sample = time.perf_counter() - t0
        pairs_full, pairs_sample = 10 * 2 * (10 + 2), 1 * 2 * (2 + 2)
        cpu = {"value": round(t_cpu_sample * pairs_full / pairs_sample, 2), "unit": "s", "cores": cgrid.threads(),
               "kind": "port", "sample": f"one outer iteration with 2 CG steps per sub-problem ({t_cpu_sample:.2f} s), "
                                         f"x {pairs_full}/{pairs_sample} NUFFT pairs"}
    print(json.dumps({
        "metric": "JSENSE coil-map estimation time (s), first echo", "value": round(t_gpu, 4), "unit": "s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(1, args.warmup), "higher_is_better": False,
        "dtype": "c64", "data": "synthetic",
        "config": {"workload": cfg.name, "coils": cfg.n_coils, "img_shape_zyx": list(cfg.img_shape),
                   "calibration_samples": int(keep.sum()), "kernel_width": 16, "calibration_width": 24,
                   "outer_iterations": 10, "cg_iterations": 10},
        "maps_shape": list(maps.shape), "cpu_baseline": cpu}), flush=True)


def main(argv=None):
    args = parse(argv)
    if args.jsense:
        run_jsense(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
