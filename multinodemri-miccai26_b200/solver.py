"""Single-GPU PDHG solver for TVM / TVME / TVMW on the b200 backend.

The state the reference keeps as CuPy arrays (``pdhg_init``, ``tvme.py:190-205``;
``tvm.py:180-186``; ``tvmw.py:378-383``) lives here as torch tensors on one
device, and every iteration runs inside ``tr_pdhg_run`` (one CUDA graph per
iteration after the first).  ``run`` reproduces ``*Reconstructor.run``:
the stopping rule, the returned extrapolated image ``u_bar``, and the
``OverflowError`` retry that shrinks the steps by 0.9 (``tvme.py:571-573``).

Step rules.  ``"reference"`` keeps the reference's sigma = tau = 1/6 for every
dual (``tvme.py:968``, ``tvm.py:991-992``, ``tvmw.py:1154``): the parity mode.
``"power"`` sets block-diagonal steps from operator norms (``power_steps``):
the data operator's norm ||W^1/2 A|| by an FP64 power iteration on the
device (``tr_power_iteration``) and known bounds of the regulariser operators.
Both rules have the same fixed points (the saddle point of the same
objective); only the path to them differs.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .nufft_backend import B200NufftBackend


STEP_RULES = ("reference", "power")

# Squared norm bounds of the stacked regulariser operator of each algorithm.  A
# forward difference with a zero last row has ||D||^2 <= 4, so: TVM the motion
# difference (4); TVME the motion difference plus the echo difference followed
# by the 3-D spatial gradient (4 + 4 * 12); TVMW the motion difference, the db1
# echo transform and the db6 spatial analysis (both norm <= 1; 2 is kept for
# the db6 tree as a margin).
REG_NORM2 = {"tvm": 4.0, "tvme": 52.0, "tvmw": 7.0}


# The power iteration approaches ||W^1/2 A|| from below (20 steps measured 0.4 %
# low on the 256 x 256 x 128 cones workload); the step rule uses the estimate
# times this margin.
NORM_MARGIN = 1.02


def power_steps(algorithm: str, data_norm: float, sigma_data: float = 0.1, data_share: float = 0.9):
    """Block-diagonal PDHG steps (sigma, tau, sigma_data) from the data norm.

    PDHG with a dual step per block (Pock & Chambolle, ICCV 2011) converges
    when tau * (sigma_data ||W^1/2 A||^2 + sigma ||K_reg||^2) < 1.  The data
    block takes ``data_share`` of that budget with a small dual step
    ``sigma_data`` (the per-mode rate of the quadratic data term is best for
    sigma_data in 0.1-0.5 with tau * sigma_data * ||A||^2 close to 1; on the
    128 x 128 x 96 TVME workload 0.1 gave the smallest tolerance and the
    result closest to a 1,500-iteration solve after 300 iterations), the
    regulariser duals the rest, 1 % short of the bound.  The reference's
    sigma = tau = 1/6 gives tau * sigma_data * ||A||^2 = ||A||^2 / 36, far
    below 1 when ||A||^2 is small.
    """
    alg = algorithm.lower()
    if alg not in REG_NORM2:
        raise ValueError(f"unknown algorithm {algorithm!r}")
    if not (data_norm > 0.0 and math.isfinite(data_norm)):
        raise ValueError(f"the data operator norm must be positive and finite, got {data_norm}")
    if not (0.0 < data_share < 1.0) or not sigma_data > 0.0:
        raise ValueError("need 0 < data_share < 1 and sigma_data > 0")
    tau = data_share / (sigma_data * data_norm * data_norm)
    sigma = (1.0 - data_share) * 0.99 / (tau * REG_NORM2[alg])
    return sigma, tau, sigma_data


@dataclass
class SolveResult:
    image: object                 # torch complex64 (B, E, Z, Y, X): u_bar
    iterations: int
    tols: list = field(default_factory=list)
    seconds: float = 0.0          # device time of the PDHG iterations (CUDA events)
    sigma: float = 1 / 6
    tau: float = 1 / 6
    sigma_data: float = 1 / 6
    step_rule: str = "reference"
    data_norm: Optional[float] = None     # ||W^1/2 A|| of the power rule
    setup_seconds: float = 0.0            # device time of the norm estimate (power rule)


class PdhgSolver:
    """Holds the plan, the sorted k-space and the PDHG state of one problem.

    ``ksp``: per bin (E, C, M_b) or (E, C, TR_b, RO) arrays; ``coords``: per
    bin (..., 3) zyx grid units; ``dcf``: per bin weights; ``mps``: (C, Z, Y, X).
    """

    def __init__(self, algorithm: str, img_shape: Sequence[int], coords, dcf, mps, ksp, *, device=0,
                 l2_coupling: bool = False, sigma: float = 1 / 6, tau: float = 1 / 6, lam_m: float = 1e-5,
                 lam_e: float = 1e-5, lam_w1: float = 1e-5, lam_w2: float = 1e-5, use_graph: bool = True,
                 backend: Optional[B200NufftBackend] = None, autotune: bool = True, step_rule: str = "reference",
                 power_iters: int = 20):
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
        if step_rule not in STEP_RULES:
            raise ValueError(f"step_rule must be one of {STEP_RULES}, got {step_rule!r}")
        self.step_rule = step_rule
        self.power_iters = int(power_iters)
        self.sigma, self.tau = float(sigma), float(tau)
        self.sigma_data = self.sigma
        self.data_norm = None
        self.setup_seconds = 0.0
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
        if self.step_rule == "power":
            self.set_power_steps()

    def set_power_steps(self, n_iter: Optional[int] = None, sigma_data: float = 0.1, data_share: float = 0.9):
        """Estimate ||W^1/2 A|| on the device (FP64 power iteration on one image
        per bin, in the first B images of the state ``g`` as scratch) and set
        the block-diagonal steps of ``power_steps`` from the estimate times
        ``NORM_MARGIN``; the device time goes to ``setup_seconds``."""
        torch = self.torch
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gen = torch.Generator(device=self.device)
        gen.manual_seed(0)
        shape = (self.B,) + self.img_shape
        with torch.cuda.device(self.device), torch.cuda.stream(self.stream):
            start.record(self.stream)
            work = self.g.view(-1)[: self.B * int(np.prod(self.img_shape))].view(shape)
            work.copy_(torch.randn(shape, dtype=torch.complex64, device=self.device, generator=gen))
            self.data_norm = self.backend.power_norm(self.power_iters if n_iter is None else int(n_iter), work=work)
            stop.record(self.stream)
            self.g.zero_()
        stop.synchronize()
        self.setup_seconds = start.elapsed_time(stop) / 1e3
        self.sigma, self.tau, self.sigma_data = power_steps(self.algorithm, self.data_norm * NORM_MARGIN, sigma_data,
                                                            data_share)
        self.step_rule = "power"

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

    def _params(self, sigma, tau, sigma_data=None) -> _lib.PdhgParams:
        pr = _lib.PdhgParams()
        pr.algorithm = _lib.TR_ALG[self.algorithm]
        pr.l2_coupling = int(self.l2_coupling)
        pr.sigma, pr.tau = sigma, tau
        pr.sigma_data = sigma if sigma_data is None else sigma_data
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
    def iterate(self, n_iter: int, tol: float = 0.0, sigma: float | None = None, tau: float | None = None,
                sigma_data: float | None = None):
        """Run up to n_iter iterations from the current state; returns (iters, tols).
        Steps default to the solver's (``sigma_data`` follows an explicit
        ``sigma`` unless given)."""
        torch = self.torch
        hist = (ctypes.c_double * max(1, n_iter))()
        done = ctypes.c_int32(0)
        if sigma_data is None:
            sigma_data = self.sigma_data if sigma is None else sigma
        st, pr = self._state_struct(), self._params(self.sigma if sigma is None else sigma,
                                                     self.tau if tau is None else tau, sigma_data)
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
        sigma, tau, sigma_data = self.sigma, self.tau, self.sigma_data
        while True:
            self.reset(init)
            start = torch.cuda.Event(enable_timing=True)
            stop = torch.cuda.Event(enable_timing=True)
            try:
                start.record(self.stream)
                iters, tols = self.iterate(max_iter, tol, sigma, tau, sigma_data)
                stop.record(self.stream)
                stop.synchronize()
                return SolveResult(image=self.u_bar, iterations=iters, tols=tols,
                                   seconds=start.elapsed_time(stop) / 1e3, sigma=sigma, tau=tau,
                                   sigma_data=sigma_data, step_rule=self.step_rule, data_norm=self.data_norm,
                                   setup_seconds=self.setup_seconds)
            except OverflowError:
                if self.algorithm == "tvmw":   # the reference's TVMW has no retry
                    raise
                sigma *= 0.9
                tau *= 0.9
                sigma_data *= 0.9

    def close(self):
        self.backend.close()
