"""Bin-sharded PDHG over several GPUs: one process per GPU, motion bins split.

The reference spreads the motion x echo grid over MPI ranks and exchanges
one-bin ghosts around the motion TV (``tvme.py:217-229`` sends u_bar forward,
``tvme.py:421-437`` needs p_m of the previous bin; ``tvm.py:230-260``,
``tvm.py:342-357``, ``tvmw.py:662-670`` likewise) and all-reduces the two
stopping sums (``tvme.py:518-551``).  Here every rank holds a contiguous range
of motion bins (all echoes and coils of them) in one plan; an iteration is

    u_bar halo   first local u_bar bin -> previous rank (its ``u_bar_next``),
                 posted without waiting
    phase 1a     data dual (forward NUFFTs), TVMW wavelet dual: local state only,
                 so it runs while the halo travels           (tr_pdhg_phase 3)
    (wait for the u_bar halo)
    phase 1b     TV / W1 duals, data gradient                (tr_pdhg_phase 4)
    p_m halo     last local p_m bin -> next rank (its ``p_m_prev``)
    phase 2      primal update, extrapolation, local FP64 stopping sums
    all-reduce   of the two sums; every rank takes the same stopping decision

The orchestration (``ShardedPdhg``) only needs an engine with those phases
and a communicator; ``B200ShardEngine`` is the GPU engine (NCCL between
ranks), and the same orchestration runs over gloo on CPU in the tests.
Ranks without bins (more ranks than bins) take part in the all-reduce only.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib


# ---------------------------------------------------------------------- partition
def partition_bins(counts: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Contiguous bin ranges [start, end) per rank minimising the largest
    per-rank sample count (exact dynamic programme; uneven bins allowed).
    With more ranks than bins the trailing ranks get empty ranges."""
    counts = [int(c) for c in counts]
    B = len(counts)
    if world < 1:
        raise ValueError("world must be >= 1")
    parts = min(world, B)
    pref = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    INF = np.iinfo(np.int64).max
    # best[k][j]: minimal max-load of the first j bins over k ranks (each >= 1 bin)
    best = np.full((parts + 1, B + 1), INF, dtype=np.int64)
    cut = np.zeros((parts + 1, B + 1), dtype=np.int64)
    best[0][0] = 0
    for k in range(1, parts + 1):
        for j in range(k, B + 1):
            for i in range(k - 1, j):
                if best[k - 1][i] == INF:
                    continue
                load = max(best[k - 1][i], pref[j] - pref[i])
                if load < best[k][j]:
                    best[k][j] = load
                    cut[k][j] = i
    ranges = []
    j = B
    for k in range(parts, 0, -1):
        i = int(cut[k][j])
        ranges.append((i, j))
        j = i
    ranges.reverse()
    ranges += [(B, B)] * (world - parts)
    return ranges


def neighbours(ranges: Sequence[Tuple[int, int]], rank: int) -> Tuple[Optional[int], Optional[int]]:
    """Previous and next rank holding bins (None at the ends or for an idle rank)."""
    if ranges[rank][0] == ranges[rank][1]:
        return None, None
    active = [r for r, (a, b) in enumerate(ranges) if b > a]
    i = active.index(rank)
    prev = active[i - 1] if i > 0 else None
    nxt = active[i + 1] if i + 1 < len(active) else None
    return prev, nxt


# ---------------------------------------------------------------------- communication
class TorchHaloComm:
    """Halo passing and the stopping-sum all-reduce over ``torch.distributed``
    (NCCL with device tensors between GPUs, gloo with host tensors on CPU)."""

    def __init__(self, ranges: Sequence[Tuple[int, int]], group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.prev, self.next = neighbours(ranges, self.rank)

    def _post(self, send, send_to, recv, recv_from):
        dist = self.dist
        ops = []
        if send_to is not None:
            ops.append(dist.P2POp(dist.isend, send, send_to, self.group))
        if recv_from is not None:
            ops.append(dist.P2POp(dist.irecv, recv, recv_from, self.group))
        return dist.batch_isend_irecv(ops) if ops else []

    def _exchange(self, send, send_to, recv, recv_from):
        self.wait(self._post(send, send_to, recv, recv_from))

    @staticmethod
    def wait(works):
        """Complete posted transfers (with NCCL: the current stream waits for them)."""
        for w in works:
            w.wait()

    def post_backward(self, first_bin, halo_next):
        """Start ``pass_backward`` and return its handle for ``wait``."""
        return self._post(first_bin, self.prev, halo_next, self.next)

    def pass_backward(self, first_bin, halo_next):
        """Send this rank's first bin to the previous rank; receive the next
        rank's first bin into ``halo_next``."""
        self._exchange(first_bin, self.prev, halo_next, self.next)

    def pass_forward(self, last_bin, halo_prev):
        """Send this rank's last bin to the next rank; receive the previous
        rank's last bin into ``halo_prev``."""
        self._exchange(last_bin, self.next, halo_prev, self.prev)

    def all_reduce_sum(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)


# ---------------------------------------------------------------------- orchestration
@dataclass
class ShardedResult:
    image: object                 # this rank's u_bar bins
    iterations: int
    tols: list = field(default_factory=list)
    seconds: float = 0.0          # device time of the iterations on this rank (CUDA events), 0 on CPU
    sigma: float = 1 / 6
    tau: float = 1 / 6


def tolerance_from(algorithm: str, num: float, den: float) -> float:
    """The reference's stopping quantity from the global sums (tvme.py:518-551;
    TVMW divides by max(||u_bar_prev||, 1e-12), tvmw.py:721-769)."""
    if not (math.isfinite(num) and math.isfinite(den)):
        return math.inf
    if algorithm == "tvmw":
        return math.sqrt(max(num, 0.0)) / max(math.sqrt(max(den, 0.0)), 1e-12)
    return math.sqrt(max(num, 0.0)) / math.sqrt(den) if den > 0 else math.inf


class ShardedPdhg:
    """``*Reconstructor.run`` over bin-sharded ranks (see the module docstring)."""

    def __init__(self, engine, comm, algorithm: str):
        self.engine = engine
        self.comm = comm
        self.algorithm = algorithm.lower()

    def iterate(self, n_iter: int, tol: float, sigma: float, tau: float):
        eng, comm = self.engine, self.comm
        tols = []
        for _ in range(n_iter):
            halo = comm.post_backward(eng.first_u_bar(), eng.u_bar_next)
            eng.phase1a(sigma, tau)                  # overlaps the u_bar halo
            comm.wait(halo)
            eng.phase1b(sigma, tau)
            comm.pass_forward(eng.last_p_m(), eng.p_m_prev)
            sums = eng.phase2(sigma, tau)
            comm.all_reduce_sum(sums)
            num, den = (float(v) for v in sums.tolist())
            if not (math.isfinite(num) and math.isfinite(den)):
                raise OverflowError("non-finite value in the tolerance reduction")
            t = tolerance_from(self.algorithm, num, den)
            tols.append(t)
            if t < tol:
                break
        return len(tols), tols

    def run(self, max_iter: int = 300, tol: float = 1e-3, init: Optional[dict] = None,
            sigma: float = 1 / 6, tau: float = 1 / 6) -> ShardedResult:
        while True:
            self.engine.reset(init)
            timer = self.engine.timer()
            try:
                timer.start()
                iters, tols = self.iterate(max_iter, tol, sigma, tau)
                secs = timer.stop()
                return ShardedResult(image=self.engine.image(), iterations=iters, tols=tols, seconds=secs,
                                     sigma=sigma, tau=tau)
            except OverflowError:
                if self.algorithm == "tvmw":      # the reference's TVMW has no retry
                    raise
                sigma *= 0.9
                tau *= 0.9


# ---------------------------------------------------------------------- GPU engine
class _EventTimer:
    def __init__(self, torch, stream):
        self.torch, self.stream = torch, stream

    def start(self):
        self.a = self.torch.cuda.Event(enable_timing=True)
        self.b = self.torch.cuda.Event(enable_timing=True)
        self.a.record(self.stream)

    def stop(self) -> float:
        self.b.record(self.stream)
        self.b.synchronize()
        return self.a.elapsed_time(self.b) / 1e3


class B200ShardEngine:
    """This rank's bins on its GPU: a ``PdhgSolver`` over the local bins plus
    the two halo buffers, driven through ``tr_pdhg_phase``.  Halo passing and
    the all-reduce run on torch's current stream, ordered against the solver's
    stream with stream waits."""

    def __init__(self, solver, bin_offset: int, n_bins_global: int):
        import torch
        self.torch = torch
        self.s = solver
        self.bin_offset = int(bin_offset)
        self.n_bins_global = int(n_bins_global)
        shp = (solver.E,) + solver.img_shape
        has_next = self.bin_offset + solver.B < self.n_bins_global
        has_prev = self.bin_offset > 0
        dev = solver.device
        self.u_bar_next = torch.zeros(shp, dtype=torch.complex64, device=dev) if has_next else None
        self.p_m_prev = torch.zeros(shp, dtype=torch.complex64, device=dev) if has_prev else None
        self.sums = torch.zeros(2, dtype=torch.float64, device=dev)
        self.shard = _lib.PdhgShard()
        self.shard.n_bins_global = self.n_bins_global
        self.shard.bin_offset = self.bin_offset
        self.shard.u_bar_next = ctypes.c_void_p(self.u_bar_next.data_ptr()) if has_next else None
        self.shard.p_m_prev = ctypes.c_void_p(self.p_m_prev.data_ptr()) if has_prev else None

    # halo views (contiguous (E, Z, Y, X) bins of the state)
    def first_u_bar(self):
        self._to_current()
        return self.s.u_bar[0]

    def last_p_m(self):
        self._to_current()
        return self.s.p_m[-1]

    def _to_current(self):
        self.torch.cuda.current_stream(self.s.device).wait_stream(self.s.stream)

    def _to_solver(self):
        self.s.stream.wait_stream(self.torch.cuda.current_stream(self.s.device))

    def reset(self, init):
        self.s.reset(init)

    def timer(self):
        return _EventTimer(self.torch, self.s.stream)

    def _phase(self, phase: int, sigma: float, tau: float):
        self._to_solver()
        st, pr = self.s._state_struct(), self.s._params(sigma, tau)
        rc = _lib.load().tr_pdhg_phase(self.s.backend.plan, ctypes.byref(st), ctypes.byref(pr),
                                       ctypes.byref(self.shard), int(phase),
                                       ctypes.c_void_p(self.sums.data_ptr()),
                                       ctypes.c_void_p(self.s.stream.cuda_stream))
        _lib.check(rc, "tr_pdhg_phase")

    def phase1(self, sigma, tau):
        self._phase(1, sigma, tau)

    def phase1a(self, sigma, tau):
        self._phase(3, sigma, tau)

    def phase1b(self, sigma, tau):
        self._phase(4, sigma, tau)

    def phase2(self, sigma, tau):
        self._phase(2, sigma, tau)
        self._to_current()
        return self.sums

    def image(self):
        self._to_current()
        return self.s.u_bar


class IdleEngine:
    """A rank without bins (more ranks than bins): joins the all-reduce with zero sums."""

    u_bar_next = None
    p_m_prev = None

    def __init__(self, device):
        import torch
        self.torch = torch
        self.device = torch.device(device)
        self.sums = torch.zeros(2, dtype=torch.float64, device=self.device)

    def first_u_bar(self):
        return None

    def last_p_m(self):
        return None

    def reset(self, init):
        pass

    def timer(self):
        return _EventTimer(self.torch, self.torch.cuda.current_stream(self.device))

    def phase1(self, sigma, tau):
        pass

    def phase1a(self, sigma, tau):
        pass

    def phase1b(self, sigma, tau):
        pass

    def phase2(self, sigma, tau):
        self.sums.zero_()
        return self.sums

    def image(self):
        return None


def local_problem(ranges, rank, coords, dcf, ksp):
    """This rank's slice of per-bin lists and its (offset, count) of bins."""
    a, b = ranges[rank]
    return coords[a:b], dcf[a:b], ksp[a:b], a, b - a
