"""CPU restatement of the TVMW wavelet operators (test oracle).

* W1: the level-1 db1 (Haar) pair along the echo axis exactly as written in the
  reference, ``algorithms/tvmw.py:312-343`` (forward) and ``:345-375``
  (adjoint), collapsed onto one device (zero ghosts past both global ends).
* W2: PyWavelets-convention, ``mode="zero"`` db6 ``wavedec3`` / ``waverec3``.
  The reference obtains these from ptwt (``algorithms/tvmw.py:196-206``,
  unpinned, ``environment.yml:17``), which follows PyWavelets' lengths and
  coefficient layout.  ptwt / PyWavelets are absent here, so this restates the
  published algorithm:
  - Daubechies extremal-phase filters by spectral factorisation of
    ``P(y) = sum_k C(N-1+k, k) y^k`` (Daubechies 1988);
  - analysis ``c[o] = sum_j f[j] x[2o+1-j]`` with zero extension, output
    length ``floor((n + F - 1) / 2)``;
  - synthesis (upsample by two, convolve, keep the valid part) with output
    length ``2n - F + 2``; a reconstructed approximation that is one longer
    than the next level's details is cropped to them;
  - ``level=None`` -> ``min_axis floor(log2(n / (F - 1)))``.
  Parity against ptwt itself is unpinned; perfect reconstruction holds.
"""

from __future__ import annotations

import itertools
import math
from functools import lru_cache
from typing import Sequence

import numpy as np


@lru_cache(maxsize=None)
def daubechies_rec_lo(n_vanishing: int) -> np.ndarray:
    """Reconstruction low-pass filter of dbN in PyWavelets order (length 2N)."""
    N = int(n_vanishing)
    if N == 1:
        return np.array([1.0, 1.0]) / math.sqrt(2.0)
    # P(y) = sum_{k<N} C(N-1+k, k) y^k ; roots in y, mapped to z, keep |z| < 1.
    coeffs = [math.comb(N - 1 + k, k) for k in range(N)]
    y_roots = np.roots(coeffs[::-1])
    z_roots = []
    for y in y_roots:
        b = 1.0 - 2.0 * y
        disc = np.sqrt(b * b - 1.0 + 0j)
        z1, z2 = b + disc, b - disc
        z_roots.append(z1 if abs(z1) < 1.0 else z2)
    poly = np.array([1.0 + 0j])
    for _ in range(N):
        poly = np.convolve(poly, [1.0, 1.0])
    for z in z_roots:
        poly = np.convolve(poly, [1.0, -z])
    h = np.real(poly)
    h = h * (math.sqrt(2.0) / h.sum())
    # PyWavelets' rec_lo starts with the small positive leading tap of the
    # extremal-phase filter (db2: 0.483, 0.837, 0.224, -0.129).
    if abs(h[0]) < abs(h[-1]):
        h = h[::-1]
    return h.copy()


def filter_bank(name: str):
    """(dec_lo, dec_hi, rec_lo, rec_hi) in PyWavelets conventions."""
    if not name.startswith("db"):
        raise ValueError(f"unsupported wavelet {name!r}")
    rec_lo = daubechies_rec_lo(int(name[2:]))
    L = rec_lo.size
    dec_lo = rec_lo[::-1].copy()
    dec_hi = np.array([(-1.0) ** (k + 1) * dec_lo[L - 1 - k] for k in range(L)])
    rec_hi = dec_hi[::-1].copy()
    return dec_lo, dec_hi, rec_lo, rec_hi


def dwt_len(n: int, F: int) -> int:
    return (n + F - 1) // 2


def idwt_len(n: int, F: int) -> int:
    return 2 * n - F + 2


def max_level(shape: Sequence[int], F: int) -> int:
    levels = []
    for n in shape:
        if n < F - 1:
            levels.append(0)
        else:
            levels.append(int(math.floor(math.log2(n / (F - 1)))))
    return max(0, min(levels))


def dwt_axis(x: np.ndarray, axis: int, f: np.ndarray) -> np.ndarray:
    """Zero-mode stride-2 analysis along ``axis``: out[o] = sum_j f[j] x[2o+1-j]."""
    x = np.moveaxis(np.asarray(x), axis, -1)
    n = x.shape[-1]
    F = f.size
    n_out = dwt_len(n, F)
    xp = np.zeros(x.shape[:-1] + (n + 2 * F,), dtype=np.result_type(x.dtype, np.float64))
    xp[..., F:F + n] = x  # xp[F + m] = x[m]
    out = np.zeros(x.shape[:-1] + (n_out,), dtype=xp.dtype)
    o = np.arange(n_out)
    for j in range(F):
        out += f[j] * xp[..., F + 2 * o + 1 - j]
    return np.moveaxis(out, -1, axis)


def idwt_axis(ca: np.ndarray | None, cd: np.ndarray | None, axis: int, f_lo: np.ndarray,
              f_hi: np.ndarray) -> np.ndarray:
    """Zero-mode synthesis along ``axis`` (valid part of upsample-then-convolve)."""
    ref = ca if ca is not None else cd
    n = ref.shape[axis]
    F = f_lo.size
    n_out = idwt_len(n, F)
    parts = []
    for c, f in ((ca, f_lo), (cd, f_hi)):
        if c is None:
            continue
        cc = np.moveaxis(np.asarray(c), axis, -1)
        out = np.zeros(cc.shape[:-1] + (n_out,), dtype=np.result_type(cc.dtype, np.float64))
        i = np.arange(F // 2 - 1, n)
        o = 2 * (i - (F // 2 - 1))
        for j in range(F // 2):
            out[..., o] += f[2 * j] * cc[..., i - j]
            out[..., o + 1] += f[2 * j + 1] * cc[..., i - j]
        parts.append(out)
    total = parts[0] if len(parts) == 1 else parts[0] + parts[1]
    return np.moveaxis(total, -1, axis)


def dwtn(x: np.ndarray, name: str, axes=(-3, -2, -1)) -> dict:
    dec_lo, dec_hi, _, _ = filter_bank(name)
    coeffs = {"": np.asarray(x)}
    for ax in axes:
        nxt = {}
        for key, arr in coeffs.items():
            nxt[key + "a"] = dwt_axis(arr, ax, dec_lo)
            nxt[key + "d"] = dwt_axis(arr, ax, dec_hi)
        coeffs = nxt
    return coeffs


def idwtn(coeffs: dict, name: str, axes=(-3, -2, -1)) -> np.ndarray:
    _, _, rec_lo, rec_hi = filter_bank(name)
    cur = dict(coeffs)
    nd = len(axes)
    for depth in range(nd - 1, -1, -1):
        ax = axes[depth]
        nxt = {}
        for prefix in ("".join(p) for p in itertools.product("ad", repeat=depth)):
            nxt[prefix] = idwt_axis(cur.get(prefix + "a"), cur.get(prefix + "d"), ax, rec_lo, rec_hi)
        cur = nxt
    return cur[""]


DETAIL_KEYS = tuple("".join(p) for p in itertools.product("ad", repeat=3) if "".join(p) != "aaa")


def wavedec3(x: np.ndarray, name: str = "db6", level: int | None = None, axes=(-3, -2, -1)) -> list:
    """[cA_L, {details level L}, ..., {details level 1}] like PyWavelets/ptwt."""
    F = filter_bank(name)[0].size
    shape = [np.asarray(x).shape[a] for a in axes]
    if level is None:
        level = max_level(shape, F)
    a = np.asarray(x)
    details = []
    for _ in range(level):
        c = dwtn(a, name, axes)
        a = c.pop("aaa")
        details.append(c)
    return [a] + details[::-1]


def waverec3(coeffs: list, name: str = "db6", axes=(-3, -2, -1)) -> np.ndarray:
    a = coeffs[0]
    for d in coeffs[1:]:
        dshape = d[DETAIL_KEYS[0]].shape
        sl = tuple(slice(0, dshape[ax]) for ax in range(len(dshape)))
        a = a[sl]
        full = dict(d)
        full["aaa"] = a
        a = idwtn(full, name, axes)
    return a


def coeff_shapes(shape_zyx: Sequence[int], name: str = "db6", level: int | None = None) -> list:
    """Per-level subband shapes (coarsest first), matching ``wavedec3``."""
    F = filter_bank(name)[0].size
    if level is None:
        level = max_level(shape_zyx, F)
    shapes = []
    cur = list(shape_zyx)
    for _ in range(level):
        cur = [dwt_len(n, F) for n in cur]
        shapes.append(tuple(cur))
    return shapes[::-1]


# --------------------------------------------------------------------------
# W1: Haar along the echo axis (reference tvmw.py:312-375), single device.
# --------------------------------------------------------------------------

def w1_forward(u: np.ndarray) -> np.ndarray:
    """u (B, E, ...) -> coeff; even e: (x_e + x_{e+1})/sqrt2, odd e: (x_e - x_{e-1})/sqrt2."""
    E = u.shape[1]
    s = 1.0 / math.sqrt(2.0)
    out = np.zeros_like(u)
    for e in range(E):
        if e % 2 == 0:
            x1 = u[:, e + 1] if e + 1 < E else 0.0
            out[:, e] = (u[:, e] + x1) * s
        else:
            out[:, e] = (-u[:, e - 1] + u[:, e]) * s
    return out


def w1_adjoint(p: np.ndarray) -> np.ndarray:
    """Adjoint: even e: (a_e - d_{e+1})/sqrt2, odd e: (a_{e-1} + d_e)/sqrt2."""
    E = p.shape[1]
    s = 1.0 / math.sqrt(2.0)
    out = np.zeros_like(p)
    for e in range(E):
        if e % 2 == 0:
            dn = p[:, e + 1] if e + 1 < E else 0.0
            out[:, e] = (p[:, e] - dn) * s
        else:
            out[:, e] = (p[:, e - 1] + p[:, e]) * s
    return out
