"""Bin-sharded PDHG orchestration over gloo (CPU, world sizes 2-4).

Each rank runs the oracle's PDHG arithmetic on its contiguous range of motion
bins (``tests/_shard_oracle.py``) through ``parallel.ShardedPdhg`` and
``parallel.TorchHaloComm``: halo passing of u_bar and p_m and the all-reduce
of the stopping sums.  The gathered images and tolerances must equal the
single-process oracle run on the same golden problem.
"""

from __future__ import annotations

import os
import socket
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

from tests._fixtures import load_golden, oracle_problem, pkg  # noqa: E402


def test_partition_bins_balanced_and_contiguous():
    par = pkg("parallel")
    counts = [5, 1, 1, 1, 8, 2, 2]
    for world in range(1, 9):
        ranges = par.partition_bins(counts, world)
        assert len(ranges) == world
        covered = [b for a, e in ranges for b in range(a, e)]
        assert covered == list(range(len(counts)))
        for (a0, e0), (a1, e1) in zip(ranges, ranges[1:]):
            assert e0 == a1
        if world <= len(counts):
            assert all(e > a for a, e in ranges)
    # the optimum for two ranks of [5, 1, 1, 1, 8, 2, 2]: [5,1,1,1] | [8,2,2] -> max 12
    r = par.partition_bins(counts, 2)
    assert max(sum(counts[a:e]) for a, e in r) == 12
    assert par.partition_bins([3, 3], 4)[2:] == [(2, 2), (2, 2)]


def test_neighbours_skip_idle_ranks():
    par = pkg("parallel")
    ranges = [(0, 2), (2, 3), (3, 3), (3, 3)]
    assert par.neighbours(ranges, 0) == (None, 1)
    assert par.neighbours(ranges, 1) == (0, None)
    assert par.neighbours(ranges, 2) == (None, None)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, name, n_iter, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from tests._shard_oracle import IdleEngine, OracleShardEngine
        par = pkg("parallel")
        fx = load_golden(name)
        pb = oracle_problem(fx)
        counts = [k.shape[-1] for k in pb.ksp]
        ranges = par.partition_bins(counts, world)
        a, e = ranges[rank]
        if e > a:
            from oracle import pdhg as op
            local = op.Problem(nufft=_SubNufft(pb.nufft, a), ksp=pb.ksp[a:e], dcf=pb.dcf[a:e], mps=pb.mps,
                               dtype=pb.dtype)
            eng = OracleShardEngine(local, name, a, len(counts), lam=float(fx["lam"]), l2_coupling=bool(fx["l2"]))
        else:
            eng = IdleEngine()
        comm = par.TorchHaloComm(ranges)
        res = par.ShardedPdhg(eng, comm, name).run(max_iter=n_iter, tol=0.0)
        np.savez(Path(outdir) / f"rank{rank}.npz", a=a, e=e, tols=np.array(res.tols),
                 image=res.image if res.image is not None else np.zeros(0))
    finally:
        dist.destroy_process_group()


class _SubNufft:
    """The oracle NUFFT of a problem restricted to bins [offset, ...)."""

    def __init__(self, nf, offset):
        self.nf, self.offset = nf, offset

    def forward(self, image, b):
        return self.nf.forward(image, b + self.offset)

    def adjoint(self, ksp, b):
        return self.nf.adjoint(ksp, b + self.offset)


@pytest.mark.parametrize("name,world", [("tvm", 2), ("tvme", 2), ("tvme", 3), ("tvme", 4), ("tvmw", 2)])
def test_sharded_pdhg_matches_single_process(name, world):
    import torch.multiprocessing as mp
    from oracle import pdhg as op
    n_iter = 4
    fx = load_golden(name)
    pb = oracle_problem(fx)
    lam = float(fx["lam"])
    ref = op.run(name, pb, max_iter=n_iter, tol=0.0, lam_m=lam, lam_e=lam, lam1=lam, lam2=lam, lam3=lam,
                 l2_coupling=bool(fx["l2"]))
    with tempfile.TemporaryDirectory() as td:
        mp.spawn(_rank_main, args=(world, _free_port(), name, n_iter, td), nprocs=world, join=True)
        parts, tols = [], None
        for r in range(world):
            z = np.load(Path(td) / f"rank{r}.npz")
            if int(z["e"]) > int(z["a"]):
                parts.append((int(z["a"]), z["image"]))
            tols = z["tols"] if tols is None else tols
            np.testing.assert_array_equal(z["tols"], tols)      # every rank saw the same stopping sums
    img = np.concatenate([p for _, p in sorted(parts, key=lambda t: t[0])])
    rel = np.linalg.norm(img - ref.image) / np.linalg.norm(ref.image)
    assert rel < 1e-12, rel
    np.testing.assert_allclose(tols, ref.tols, rtol=1e-9)
