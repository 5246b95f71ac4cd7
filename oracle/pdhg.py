"""CPU restatement of the reference PDHG loops on one device (test oracle).

Follows, operation by operation, with every rank's ``is_*_first/last`` flag
true (one device holds all bins and echoes, so every ghost is a global edge):

* TVM   ``algorithms/tvm.py:227-380`` (iteration) and ``:390-491`` (run/stop)
* TVME  ``algorithms/tvme.py:208-482`` (iteration) and ``:496-575`` (run/stop)
* TVMW  ``algorithms/tvmw.py:385-685`` (iteration) and ``:698-786`` (run/stop)

The NUFFT is any object with ``forward(images (..., Z, Y, X), bin) -> (..., M_b)``
and ``adjoint(ksp (..., M_b), bin) -> (..., Z, Y, X)`` (the reference's
``NufftBackend`` contract, ``nufft_backend.py:38-44``, batched over leading
axes).  ``dtype`` selects complex128 (the FP64 oracle) or complex64.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import nufft as _nf
from . import wavelets as _wv


class OracleNufft:
    """Per-bin KB NUFFT from ``oracle.nufft`` (SigPy 0.1.27 restated)."""

    def __init__(self, img_shape, coords, out_dtype=np.complex128):
        self.img_shape = tuple(int(v) for v in img_shape)
        self.coords = [np.asarray(c, dtype=np.float32) for c in coords]
        self.out_dtype = out_dtype

    @property
    def num_bins(self):
        return len(self.coords)

    def forward(self, image, b):
        return _nf.nufft(image, self.coords[b]).astype(self.out_dtype)

    def adjoint(self, ksp, b):
        return _nf.nufft_adjoint(ksp, self.coords[b], self.img_shape).astype(self.out_dtype)


# ---------------------------------------------------------------- differences
def dxf(x):
    d = np.zeros_like(x)
    d[..., :-1] = x[..., 1:] - x[..., :-1]
    return d


def dyf(x):
    d = np.zeros_like(x)
    d[..., :-1, :] = x[..., 1:, :] - x[..., :-1, :]
    return d


def dzf(x):
    d = np.zeros_like(x)
    d[..., :-1, :, :] = x[..., 1:, :, :] - x[..., :-1, :, :]
    return d


def dxb(x):
    """Exact transpose of ``dxf`` (tvme.py:171-175)."""
    d = np.zeros_like(x)
    d[..., :-1] = -x[..., :-1]
    d[..., 1:] = -d[..., :-1] + d[..., 1:]
    return d


def dyb(x):
    d = np.zeros_like(x)
    d[..., :-1, :] = -x[..., :-1, :]
    d[..., 1:, :] = -d[..., :-1, :] + d[..., 1:, :]
    return d


def dzb(x):
    d = np.zeros_like(x)
    d[..., :-1, :, :] = -x[..., :-1, :, :]
    d[..., 1:, :, :] = -d[..., :-1, :, :] + d[..., 1:, :, :]
    return d


def motion_diff(u):
    d = np.zeros_like(u)
    if u.shape[0] > 1:
        d[:-1] = u[1:] - u[:-1]
    d[-1] = 0
    return d


def motion_div_tvme(p):
    """tvme.py:421-437 with is_motion_first = is_motion_last = True; returns D_m^T p."""
    B = p.shape[0]
    d = np.zeros_like(p)
    if B > 1:
        d[1:] = p[:-1] - p[1:]
    d[0] = -p[0]
    if B > 1:
        d[-1] = p[-2]
    else:
        d[0] = 0
    return d


def echo_div_tvme(divp):
    """tvme.py:361-363, :444-454 (global first and last echo on one device)."""
    E = divp.shape[1]
    d = np.zeros_like(divp)
    if E > 1:
        d[:, 1:] = divp[:, :-1] - divp[:, 1:]
    d[:, 0] = -divp[:, 0]
    if E > 1:
        d[:, -1] = divp[:, -2]
    return d


def prox_motion(p_m, lam, l2_coupling):
    """L1: tvme.py:299-302 ; L2 over all echoes: tvme.py:285-297, :326-337."""
    if l2_coupling:
        mag = np.sqrt(np.sum(np.abs(p_m) ** 2, axis=1, keepdims=True))
        return p_m / np.maximum(1.0, mag / lam)
    return p_m / np.maximum(1.0, np.abs(p_m) / lam)


# ---------------------------------------------------------------- problem
@dataclass
class Problem:
    """Single-device PDHG inputs (all already binned and normalised)."""
    nufft: object
    ksp: list            # per bin (E, C, M_b) complex
    dcf: list            # per bin (M_b,) float
    mps: np.ndarray      # (C, Z, Y, X) complex
    dtype: type = np.complex128

    @property
    def B(self):
        return len(self.ksp)

    @property
    def E(self):
        return self.ksp[0].shape[0]

    @property
    def C(self):
        return self.mps.shape[0]

    @property
    def img_shape(self):
        return tuple(self.mps.shape[-3:])

    def cast(self):
        rdt = np.float64 if self.dtype == np.complex128 else np.float32
        self.ksp = [np.asarray(k, dtype=self.dtype) for k in self.ksp]
        self.dcf = [np.asarray(d, dtype=rdt) for d in self.dcf]
        self.mps = np.asarray(self.mps, dtype=self.dtype)
        return self


def data_dual(pb: Problem, u_bar, q, sigma):
    """q[b] <- (q[b] + sigma (F_b(u_bar[b,e] S_c) - y[b][e][c])) / (1 + sigma)."""
    for b in range(pb.B):
        img = u_bar[b][:, None] * pb.mps[None]            # (E, C, Z, Y, X)
        tmp = pb.nufft.forward(img, b).astype(pb.dtype) - pb.ksp[b]
        q[b] = (q[b] + sigma * tmp) / (1 + sigma)
    return q


def data_grad(pb: Problem, q):
    """g[b,e] = sum_c conj(S_c) F_b^H(dcf_b q[b][e][c])."""
    out = np.zeros((pb.B, pb.E) + pb.img_shape, dtype=pb.dtype)
    mconj = np.conj(pb.mps)
    for b in range(pb.B):
        x = pb.nufft.adjoint(pb.dcf[b] * q[b], b).astype(pb.dtype)  # (E, C, Z, Y, X)
        out[b] = np.sum(x * mconj[None], axis=1)
    return out


# ---------------------------------------------------------------- TVM
def tvm_init(pb: Problem):
    z = np.zeros((pb.B, pb.E) + pb.img_shape, dtype=pb.dtype)
    return {"u_bar": z.copy(), "u": z.copy(), "p_m": z.copy(),
            "q": [np.zeros_like(k) for k in pb.ksp]}


def tvm_iterate(pb: Problem, st, sigma, tau, lam, l2_coupling=False, sigma_data=None):
    """One ``TvmReconstructor.pdhg`` step (tvm.py:227-380), default reduce mode.
    ``sigma_data`` (default: ``sigma``) is the data-dual step; the reference uses
    one sigma for every dual."""
    u_old = st["u"].copy()
    st["q"] = data_dual(pb, st["u_bar"], st["q"], sigma if sigma_data is None else sigma_data)
    p_m = st["p_m"] + sigma * motion_diff(st["u_bar"])
    p_m = prox_motion(p_m, lam, l2_coupling)
    g = data_grad(pb, st["q"])
    B = p_m.shape[0]
    divergence = np.zeros_like(p_m)
    if B > 1:
        divergence[1:] = p_m[1:] - p_m[:-1]
    divergence[0] = p_m[0]
    if B > 1:
        divergence[-1] = -p_m[-2]
    else:
        divergence[0] = 0
    st["u"] = st["u"] - tau * (g - divergence)
    st["u_bar"] = 2 * st["u"] - u_old
    st["p_m"] = p_m
    return st


# ---------------------------------------------------------------- TVME
def tvme_init(pb: Problem):
    st = tvm_init(pb)
    z = np.zeros_like(st["u"])
    st.update({"p_ex": z.copy(), "p_ey": z.copy(), "p_ez": z.copy()})
    return st


def tvme_iterate(pb: Problem, st, sigma, tau, lam_m, lam_e, l2_coupling=False, sigma_data=None):
    """One ``TvmeReconstructor.pdhg`` step (tvme.py:208-482) on one device."""
    u_bar = st["u_bar"]
    u_old = st["u"].copy()
    st["q"] = data_dual(pb, u_bar, st["q"], sigma if sigma_data is None else sigma_data)
    p_m = st["p_m"] + sigma * motion_diff(u_bar)
    if not l2_coupling:
        p_m = p_m / np.maximum(1.0, np.abs(p_m) / lam_m)
    diff_e = np.zeros_like(u_bar)
    if pb.E > 1:
        diff_e[:, :-1] = u_bar[:, 1:] - u_bar[:, :-1]
    diff_e[:, -1] = 0
    p_ex = st["p_ex"] + sigma * dxf(diff_e)
    p_ey = st["p_ey"] + sigma * dyf(diff_e)
    p_ez = st["p_ez"] + sigma * dzf(diff_e)
    absp = np.sqrt(np.abs(p_ex) ** 2 + np.abs(p_ey) ** 2 + np.abs(p_ez) ** 2)
    den = np.maximum(1.0, absp / lam_e)
    p_ex, p_ey, p_ez = p_ex / den, p_ey / den, p_ez / den
    if l2_coupling:
        mag = np.sqrt(np.sum(np.abs(p_m) ** 2, axis=1, keepdims=True))
        p_m = p_m / np.maximum(1.0, mag / lam_m)
    divp = dxb(p_ex) + dyb(p_ey) + dzb(p_ez)
    divp_e = echo_div_tvme(divp)
    g = data_grad(pb, st["q"])
    u = st["u"]
    u = u - tau * motion_div_tvme(p_m)
    u = u - tau * divp_e
    u = u - tau * g
    st.update({"u": u, "u_bar": 2 * u - u_old, "p_m": p_m, "p_ex": p_ex, "p_ey": p_ey, "p_ez": p_ez})
    return st


# ---------------------------------------------------------------- TVMW
def w2_project(coeffs, lam):
    """_tree_project_linf_complex2ch_ (tvmw.py:162-193) on complex coefficients."""
    def proj(c):
        if lam <= 0:
            return np.zeros_like(c)
        mag = np.sqrt(c.real * c.real + c.imag * c.imag + 1e-12)
        return c * np.minimum(lam / mag, 1.0)
    out = [proj(coeffs[0])]
    for d in coeffs[1:]:
        out.append({k: proj(v) for k, v in d.items()})
    return out


def w2_axpy(dst, a, src):
    out = [dst[0] + a * src[0]]
    for dd, ss in zip(dst[1:], src[1:]):
        out.append({k: dd[k] + a * ss[k] for k in dd})
    return out


def w2_zeros_like(c):
    return [np.zeros_like(c[0])] + [{k: np.zeros_like(v) for k, v in d.items()} for d in c[1:]]


def tvmw_init(pb: Problem):
    z = np.zeros((pb.B, pb.E) + pb.img_shape, dtype=pb.dtype)
    return {"u_bar": z.copy(), "u_old": z.copy(), "u_tmp": z.copy(), "p_m": z.copy(),
            "p_w1": z.copy(), "p_w2": [None] * pb.B, "q": [np.zeros_like(k) for k in pb.ksp]}


def tvmw_iterate(pb: Problem, st, sigma, tau, lam1, lam2, lam3, l2_coupling=False, wavelet="db6",
                 sigma_data=None):
    """One ``TvmwReconstructor.pdhg`` step (tvmw.py:385-685) on one device."""
    u = st["u_bar"]                       # "primal_u" in the reference
    st["u_old"] = st["u_tmp"].copy()
    for b in range(pb.B):
        w2 = _wv.wavedec3(u[b], wavelet)
        if st["p_w2"][b] is None:
            st["p_w2"][b] = w2_zeros_like(w2)
        st["p_w2"][b] = w2_project(w2_axpy(st["p_w2"][b], sigma, w2), lam3)
    st["q"] = data_dual(pb, u, st["q"], sigma if sigma_data is None else sigma_data)
    p_m = st["p_m"] + sigma * motion_diff(u)
    if not l2_coupling:
        p_m = p_m / np.maximum(1.0, np.abs(p_m) / lam1)
    p_w1 = st["p_w1"] + sigma * _wv.w1_forward(u)
    if lam2 > 0:
        p_w1 = p_w1 / np.maximum(1.0, np.abs(p_w1) / lam2)
    else:
        p_w1 = np.zeros_like(p_w1)
    if l2_coupling:
        mag = np.sqrt(np.sum(np.abs(p_m) ** 2, axis=1, keepdims=True))
        p_m = p_m / np.maximum(1.0, mag / lam1)
    g = data_grad(pb, st["q"])
    divp_w2 = np.zeros_like(u)
    for b in range(pb.B):
        rec = _wv.waverec3(st["p_w2"][b], wavelet)
        divp_w2[b] = rec[(slice(None),) + tuple(slice(0, n) for n in pb.img_shape)]
    divp_w1 = _wv.w1_adjoint(p_w1)
    divp_m = np.zeros_like(u)
    if pb.B > 1:
        divp_m[1:] = p_m[1:] - p_m[:-1]
    divp_m[0] = p_m[0]
    st["u_tmp"] = st["u_tmp"] - tau * (g - divp_m + divp_w1 + divp_w2)
    st["u_bar"] = 2 * st["u_tmp"] - st["u_old"]
    st["p_m"], st["p_w1"] = p_m, p_w1
    return st


# ---------------------------------------------------------------- run loops
@dataclass
class RunResult:
    image: np.ndarray
    iterations: int
    tols: list = field(default_factory=list)
    state: dict | None = None


def _tol_u(u, u_prev):
    """tvme.py:518-551: ||u_k - u_{k-1}|| / ||u_k|| (inf if not finite / zero)."""
    num2 = float(np.vdot((u - u_prev).ravel(), (u - u_prev).ravel()).real)
    den2 = float(np.vdot(u.ravel(), u.ravel()).real)
    if np.isfinite(num2) and np.isfinite(den2) and den2 > 0.0:
        return math.sqrt(max(num2, 0.0)) / math.sqrt(den2)
    return float("inf")


def _tol_w(u_new, u_prev):
    """tvmw.py:721-769: ||u_{k-1} - u_k|| / max(||u_{k-1}||, 1e-12) on u_bar."""
    d = u_prev - u_new
    num2 = float(np.vdot(d.ravel(), d.ravel()).real)
    den2 = float(np.vdot(u_prev.ravel(), u_prev.ravel()).real)
    if np.isfinite(num2) and np.isfinite(den2):
        return math.sqrt(max(num2, 0.0)) / max(math.sqrt(max(den2, 0.0)), 1e-12)
    return float("inf")


def run(algorithm: str, pb: Problem, *, sigma=1 / 6, tau=1 / 6, max_iter=300, tol=1e-3,
        lam_m=1e-5, lam_e=1e-5, lam1=1e-5, lam2=1e-5, lam3=1e-5, l2_coupling=False,
        init=None, keep_state=False, sigma_data=None) -> RunResult:
    """``*Reconstructor.run`` on one device; returns ``u_bar`` like the reference.

    ``init`` optionally overrides the zero initial state (used only to check
    warm starts; the reference always starts from zeros).  ``sigma_data``
    gives the data dual its own step (block-diagonal steps; the reference has
    one sigma).
    """
    pb.cast()
    alg = algorithm.lower()
    if alg == "tvm":
        st = tvm_init(pb)
    elif alg == "tvme":
        st = tvme_init(pb)
    elif alg == "tvmw":
        st = tvmw_init(pb)
    else:
        raise ValueError(algorithm)
    if init:
        for k, v in init.items():
            st[k] = v
    tols = []
    it_done = 0
    for it in range(max_iter):
        if alg == "tvmw":
            prev = st["u_bar"].copy()
            tvmw_iterate(pb, st, sigma, tau, lam1, lam2, lam3, l2_coupling, sigma_data=sigma_data)
            t = _tol_w(st["u_bar"], prev)
        else:
            prev = st["u"].copy()
            if alg == "tvm":
                tvm_iterate(pb, st, sigma, tau, lam_m, l2_coupling, sigma_data=sigma_data)
            else:
                tvme_iterate(pb, st, sigma, tau, lam_m, lam_e, l2_coupling, sigma_data=sigma_data)
            t = _tol_u(st["u"], prev)
        tols.append(t)
        it_done = it + 1
        if t < tol:
            break
    return RunResult(image=st["u_bar"], iterations=it_done, tols=tols, state=st if keep_state else None)


# ---------------------------------------------------------------- step rule
def power_norm(pb: Problem, n_iter: int = 30, seed: int = 0) -> float:
    """sqrt(||A^H W A||) by power iteration in FP64, A = [F_b S_c] over every
    bin, echo and coil and W the density weights: the data operator of the
    PDHG loop (``data_grad(data_dual(.))`` without the prox).  The reference
    has no such estimate (it fixes sigma = tau = 1/6, ``tvme.py:968``)."""
    pb.cast()
    rng = np.random.default_rng(seed)
    shape = (pb.B, pb.E) + pb.img_shape
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    lam = 0.0
    for _ in range(n_iter):
        x = x / np.linalg.norm(x.ravel())
        ksp = []
        for b in range(pb.B):
            img = x[b][:, None] * pb.mps[None]
            ksp.append(pb.nufft.forward(img, b).astype(np.complex128))
        x = data_grad(pb, ksp)
        lam = float(np.linalg.norm(x.ravel()))
    return math.sqrt(lam)

