"""CPU engine for the bin-sharded PDHG orchestration (test infrastructure).

Runs the oracle's PDHG arithmetic (``oracle/pdhg.py``) on one rank's
contiguous range of motion bins, with the two one-bin halos of the sharded
scheme, so that ``parallel.ShardedPdhg`` and ``parallel.TorchHaloComm`` can
be checked over gloo against the single-process oracle.  Only the tests use it.
"""

from __future__ import annotations

import numpy as np
import torch

from oracle import pdhg as op
from oracle import wavelets as wv


class _NullTimer:
    def start(self):
        pass

    def stop(self):
        return 0.0


class OracleShardEngine:
    def __init__(self, pb, algorithm, bin_offset, n_bins_global, lam=1e-5, l2_coupling=False):
        self.pb = pb.cast()
        self.alg = algorithm
        self.b0 = int(bin_offset)
        self.Bg = int(n_bins_global)
        self.lam = lam
        self.l2 = bool(l2_coupling)
        shp = (pb.E,) + pb.img_shape
        self._next = torch.zeros(shp, dtype=torch.complex128) if self.b0 + pb.B < self.Bg else None
        self._prev = torch.zeros(shp, dtype=torch.complex128) if self.b0 > 0 else None
        self.sums = torch.zeros(2, dtype=torch.float64)

    # halos as torch tensors sharing memory with numpy views
    @property
    def u_bar_next(self):
        return self._next

    @property
    def p_m_prev(self):
        return self._prev

    def first_u_bar(self):
        return torch.from_numpy(np.ascontiguousarray(self.st["u_bar"][0]))

    def last_p_m(self):
        return torch.from_numpy(np.ascontiguousarray(self.st["p_m"][-1]))

    def timer(self):
        return _NullTimer()

    def reset(self, init=None):
        pb = self.pb
        z = np.zeros((pb.B, pb.E) + pb.img_shape, dtype=pb.dtype)
        self.st = {"u": z.copy(), "u_bar": z.copy(), "p_m": z.copy(), "p_ex": z.copy(), "p_ey": z.copy(),
                   "p_ez": z.copy(), "p_w1": z.copy(), "p_w2": [None] * pb.B,
                   "q": [np.zeros_like(k) for k in pb.ksp]}

    def image(self):
        return self.st["u_bar"]

    # ------------------------------------------------------------------ phases
    def phase1(self, sigma, tau):
        self.phase1a(sigma, tau)
        self.phase1b(sigma, tau)

    def phase1a(self, sigma, tau):
        """The part of phase 1 that reads only this rank's state."""
        pb, st, lam = self.pb, self.st, self.lam
        ub = st["u_bar"]
        if self.alg == "tvmw":
            for b in range(pb.B):
                w2 = wv.wavedec3(ub[b], "db6")
                if st["p_w2"][b] is None:
                    st["p_w2"][b] = op.w2_zeros_like(w2)
                st["p_w2"][b] = op.w2_project(op.w2_axpy(st["p_w2"][b], sigma, w2), lam)
        st["q"] = op.data_dual(pb, ub, st["q"], sigma)

    def phase1b(self, sigma, tau):
        """The rest of phase 1: it reads the next rank's first u_bar bin."""
        pb, st, lam = self.pb, self.st, self.lam
        ub = st["u_bar"]
        # motion forward difference with the next rank's first bin as ghost
        d = np.zeros_like(ub)
        if pb.B > 1:
            d[:-1] = ub[1:] - ub[:-1]
        if self._next is not None:
            d[-1] = self._next.numpy() - ub[-1]
        p_m = st["p_m"] + sigma * d
        if not self.l2:
            p_m = p_m / np.maximum(1.0, np.abs(p_m) / lam)
        else:
            mag = np.sqrt(np.sum(np.abs(p_m) ** 2, axis=1, keepdims=True))
            p_m = p_m / np.maximum(1.0, mag / lam)
        st["p_m"] = p_m
        if self.alg == "tvme":
            diff_e = np.zeros_like(ub)
            if pb.E > 1:
                diff_e[:, :-1] = ub[:, 1:] - ub[:, :-1]
            p_ex = st["p_ex"] + sigma * op.dxf(diff_e)
            p_ey = st["p_ey"] + sigma * op.dyf(diff_e)
            p_ez = st["p_ez"] + sigma * op.dzf(diff_e)
            den = np.maximum(1.0, np.sqrt(np.abs(p_ex) ** 2 + np.abs(p_ey) ** 2 + np.abs(p_ez) ** 2) / lam)
            st["p_ex"], st["p_ey"], st["p_ez"] = p_ex / den, p_ey / den, p_ez / den
        if self.alg == "tvmw":
            p_w1 = st["p_w1"] + sigma * wv.w1_forward(ub)
            st["p_w1"] = p_w1 / np.maximum(1.0, np.abs(p_w1) / lam)
        st["g"] = op.data_grad(pb, st["q"])

    def phase2(self, sigma, tau):
        pb, st = self.pb, self.st
        p = st["p_m"]
        prev = np.zeros_like(p)                  # p_m of the previous global bin, per local bin
        if pb.B > 1:
            prev[1:] = p[:-1]
        if self._prev is not None:
            prev[0] = self._prev.numpy()
        gb = self.b0 + np.arange(pb.B)
        u_old = st["u"].copy()
        ub_old = st["u_bar"].copy()
        if self.alg == "tvme":
            dm = np.zeros_like(p)
            if self.Bg > 1:
                for i, g in enumerate(gb):
                    dm[i] = -p[i] if g == 0 else (prev[i] if g == self.Bg - 1 else prev[i] - p[i])
            divp = op.dxb(st["p_ex"]) + op.dyb(st["p_ey"]) + op.dzb(st["p_ez"])
            u = st["u"] - tau * dm
            u = u - tau * op.echo_div_tvme(divp)
            u = u - tau * st["g"]
        elif self.alg == "tvm":
            dv = np.zeros_like(p)
            if self.Bg > 1:
                for i, g in enumerate(gb):
                    dv[i] = p[i] if g == 0 else (-prev[i] if g == self.Bg - 1 else p[i] - prev[i])
            u = st["u"] - tau * (st["g"] - dv)
        else:
            dvm = np.zeros_like(p)
            for i, g in enumerate(gb):
                dvm[i] = p[i] if g == 0 else p[i] - prev[i]
            w2adj = np.zeros_like(p)
            for b in range(pb.B):
                rec = wv.waverec3(st["p_w2"][b], "db6")
                w2adj[b] = rec[(slice(None),) + tuple(slice(0, n) for n in pb.img_shape)]
            u = st["u"] - tau * (st["g"] - dvm + wv.w1_adjoint(st["p_w1"]) + w2adj)
        st["u"] = u
        st["u_bar"] = 2 * u - u_old
        if self.alg == "tvmw":
            dd = ub_old - st["u_bar"]
            num, den = np.vdot(dd, dd).real, np.vdot(ub_old, ub_old).real
        else:
            dd = u - u_old
            num, den = np.vdot(dd, dd).real, np.vdot(u, u).real
        self.sums = torch.tensor([float(num), float(den)], dtype=torch.float64)
        return self.sums


class IdleEngine:
    """A rank without bins: joins the all-reduce with zero sums."""

    u_bar_next = None
    p_m_prev = None

    def first_u_bar(self):
        return None

    def last_p_m(self):
        return None

    def timer(self):
        return _NullTimer()

    def reset(self, init=None):
        pass

    def phase1(self, sigma, tau):
        pass

    def phase1a(self, sigma, tau):
        pass

    def phase1b(self, sigma, tau):
        pass

    def phase2(self, sigma, tau):
        return torch.zeros(2, dtype=torch.float64)

    def image(self):
        return None
