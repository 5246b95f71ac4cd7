"""Single-GPU PDHG solver for TVM / TVME / TVMW on the b200 backend.

The state the reference keeps as CuPy arrays (``pdhg_init``, ``tvme.py:190-205``;
``tvm.py:180-186``; ``tvmw.py:378-383``) lives here as torch tensors on one
device, and every iteration runs inside ``tr_pdhg_run`` (one CUDA graph per
iteration after the first).  ``run`` reproduces ``*Reconstructor.run``:
the stopping rule, the returned extrapolated image ``u_bar``, and the
``OverflowError`` retry that shrinks sigma and tau by 0.9 (``tvme.py:571-573``).
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .nufft_backend import B200NufftBackend


@dataclass
class SolveResult:
    image: object                 # torch complex64 (B, E, Z, Y, X): u_bar
    iterations: int
    tols: list = field(default_factory=list)
    seconds: float = 0.0          # device time of the PDHG iterations (CUDA events)
    sigma: float = 1 / 6
    tau: float = 1 / 6


class PdhgSolver:
    """Holds the plan, the sorted k-space and the PDHG state of one problem.

    ``ksp``: per bin (E, C, M_b) or (E, C, TR_b, RO) arrays; ``coords``: per
    bin (..., 3) zyx grid units; ``dcf``: per bin weights; ``mps``: (C, Z, Y, X).
    """

    def __init__(self, algorithm: str, img_shape: Sequence[int], coords, dcf, mps, ksp, *, device=0,
                 l2_coupling: bool = False, sigma: float = 1 / 6, tau: float = 1 / 6, lam_m: float = 1e-5,
                 lam_e: float = 1e-5, lam_w1: float = 1e-5, lam_w2: float = 1e-5, use_graph: bool = True,
                 backend: Optional[B200NufftBackend] = None, autotune: bool = True):
        import torch
        self.torch = torch
        self.algorithm = algorithm.lower()
        if self.algorithm not in _lib.TR_ALG:
            raise ValueError(f"unknown algorithm {algorithm!r}")
        self.img_shape = tuple(int(v) for v in img_shape)
        mps_t = mps if isinstance(mps, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(mps))
        self.C = int(mps_t.shape[0])
        first = ksp[0]
        self.E = int(first.shape[0])
        self.B = len(ksp)
        self.backend = backend or B200NufftBackend(self.img_shape, coords, device, dcf=dcf, n_coils=self.C,
                                                   n_echoes=self.E, autotune=autotune)
        self.device = self.backend.device
        self.stream = torch.cuda.Stream(self.device)
        self.l2_coupling = bool(l2_coupling)
        self.sigma, self.tau = float(sigma), float(tau)
        self.lam = dict(lam_m=float(lam_m), lam_e=float(lam_e), lam_w1=float(lam_w1), lam_w2=float(lam_w2))
        self.use_graph = bool(use_graph)
        ncol = self.E * self.C
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            self.backend.set_maps(mps_t)
            self.y = torch.empty((self.backend.total_samples, ncol), dtype=torch.complex64, device=self.device)
            for b in range(self.B):
                off, cnt = self.backend.bin_offset(b), self.backend.bin_count(b)
                kb = ksp[b]
                kb = kb if isinstance(kb, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(kb))
                kb = kb.to(self.device, torch.complex64).reshape(ncol, cnt)
                self.backend.sort_kspace(kb, b, out=self.y[off:off + cnt])
        self.stream.synchronize()
        self._alloc_state()

    # ------------------------------------------------------------------ state
    def _alloc_state(self):
        torch = self.torch
        shp = (self.B, self.E) + self.img_shape
        z = lambda: torch.zeros(shp, dtype=torch.complex64, device=self.device)
        self.u, self.u_bar, self.p_m, self.g = z(), z(), z(), z()
        self.p_ex = self.p_ey = self.p_ez = self.p_w1 = self.p_w2 = self.w2adj = None
        if self.algorithm == "tvme":
            self.p_ex, self.p_ey, self.p_ez = z(), z(), z()
        if self.algorithm == "tvmw":
            self.p_w1 = z()
            self.w2adj = z()
            self.p_w2 = torch.zeros((self.B * self.E, self.backend.wavelet_coeffs), dtype=torch.complex64,
                                    device=self.device)
        self.q = torch.zeros_like(self.y)

    def reset(self, init: Optional[dict] = None):
        """Zero the state (the reference's pdhg_init), then apply optional overrides."""
        for name in ("u", "u_bar", "p_m", "g", "p_ex", "p_ey", "p_ez", "p_w1", "p_w2", "w2adj", "q"):
            t = getattr(self, name)
            if t is not None:
                t.zero_()
        if init:
            for k, v in init.items():
                getattr(self, k).copy_(v)

    def _state_struct(self) -> _lib.PdhgState:
        st = _lib.PdhgState()
        ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
        for name in ("u", "u_bar", "p_m", "p_ex", "p_ey", "p_ez", "p_w1", "p_w2", "w2adj", "q", "y", "g"):
            setattr(st, name, ptr(getattr(self, name)))
        return st

    def _params(self, sigma, tau) -> _lib.PdhgParams:
        pr = _lib.PdhgParams()
        pr.algorithm = _lib.TR_ALG[self.algorithm]
        pr.l2_coupling = int(self.l2_coupling)
        pr.sigma, pr.tau = sigma, tau
        pr.lam_m, pr.lam_e = self.lam["lam_m"], self.lam["lam_e"]
        pr.lam_w1, pr.lam_w2 = self.lam["lam_w1"], self.lam["lam_w2"]
        pr.use_graph = int(self.use_graph)
        return pr

    def adjoint_image(self):
        """Density-compensated, coil-combined adjoint sum_c S_c^H F_b^H (w y) per (bin, echo)."""
        torch = self.torch
        out = torch.empty((self.B, self.E) + self.img_shape, dtype=torch.complex64, device=self.device)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):
            for b in range(self.B):
                off, cnt = self.backend.bin_offset(b), self.backend.bin_count(b)
                self.backend.adjoint_bin(self.y[off:off + cnt], b, use_dcf=True, out=out[b])
        torch.cuda.current_stream(self.device).wait_stream(self.stream)
        return out

    def data_residual(self, u):
        """A u - y per bin in the internal k-space layout: the data dual's fixed point
        ((q + sigma r) / (1 + sigma) = q  <=>  q = r)."""
        torch = self.torch
        r = torch.empty_like(self.y)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(self.stream):
            for b in range(self.B):
                off, cnt = self.backend.bin_offset(b), self.backend.bin_count(b)
                self.backend.forward_bin(u[b], b, out=r[off:off + cnt])
            r.sub_(self.y)
        torch.cuda.current_stream(self.device).wait_stream(self.stream)
        return r

    # ------------------------------------------------------------------ iterate
    def iterate(self, n_iter: int, tol: float = 0.0, sigma: float | None = None, tau: float | None = None):
        """Run up to n_iter iterations from the current state; returns (iters, tols)."""
        torch = self.torch
        hist = (ctypes.c_double * max(1, n_iter))()
        done = ctypes.c_int32(0)
        st, pr = self._state_struct(), self._params(self.sigma if sigma is None else sigma,
                                                     self.tau if tau is None else tau)
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        status = _lib.load().tr_pdhg_run(self.backend.plan, ctypes.byref(st), ctypes.byref(pr), int(n_iter),
                                         float(tol), hist, ctypes.byref(done),
                                         ctypes.c_void_p(self.stream.cuda_stream))
        torch.cuda.current_stream(self.device).wait_stream(self.stream)
        _lib.check(status, "tr_pdhg_run")
        return int(done.value), [float(hist[i]) for i in range(done.value)]

    def run(self, max_iter: int = 300, tol: float = 1e-3, init: Optional[dict] = None) -> SolveResult:
        """``*Reconstructor.run`` on the device: reset, iterate, return u_bar."""
        torch = self.torch
        sigma, tau = self.sigma, self.tau
        while True:
            self.reset(init)
            start = torch.cuda.Event(enable_timing=True)
            stop = torch.cuda.Event(enable_timing=True)
            try:
                start.record(self.stream)
                iters, tols = self.iterate(max_iter, tol, sigma, tau)
                stop.record(self.stream)
                stop.synchronize()
                return SolveResult(image=self.u_bar, iterations=iters, tols=tols,
                                   seconds=start.elapsed_time(stop) / 1e3, sigma=sigma, tau=tau)
            except OverflowError:
                if self.algorithm == "tvmw":   # the reference's TVMW has no retry
                    raise
                sigma *= 0.9
                tau *= 0.9

    def close(self):
        self.backend.close()
