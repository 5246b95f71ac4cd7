"""CPU restatement of the Kaiser-Bessel NUFFT used by the reference (test oracle).

The reference calls SigPy 0.1.27 with its defaults
(``src/toporecon/nufft_backend.py:101-107`` forward, ``:109-116`` adjoint;
pinned at ``environment.yml:16``).  SigPy is not vendored and cannot be
installed here, so this module restates SigPy's published method:

forward(x, k)  = interp_KB( FFTc( pad_os( apod(x) / sqrt(N) ) ), scale(k) ) / w^3
adjoint(y, k)  = apod( crop( IFFTc( grid_KB(y, scale(k)) / w^3 ) ) * G / sqrt(N) )

with
* oversampling ``os = 1.25`` and kernel width ``w = 4``;
* ``beta = pi * sqrt((w / os * (os - 0.5))**2 - 0.8)`` (Beatty et al. 2005);
* the unnormalised Kaiser-Bessel window ``I0(beta * sqrt(1 - (d / (w/2))**2))``
  for ``|d| <= w/2`` (0 outside), where ``I0`` is evaluated with the
  Abramowitz & Stegun 9.8.1 / 9.8.2 rational approximations;
* taps ``ceil(k - w/2) .. floor(k + w/2)`` per axis (five taps when ``k`` is an
  integer, four otherwise), with periodic wrap onto the oversampled grid;
* coordinates in grid units ``[-n/2, n/2)`` per axis, ordered (z, y, x), and
  scaled onto the oversampled grid as ``k * ceil(os*n)/n + ceil(os*n)//2``;
* centred FFTs (``ifftshift -> fftn -> fftshift``) without normalisation and a
  centred zero-pad / crop (pad offset ``os_n//2 - n//2``);
* apodisation ``a(i) = r / sinh(r)``, ``r = sqrt(beta^2 - (pi*w*(i - n//2)/os_n)^2)``.

Net scaling: forward ~= direct NUDFT ``sum_r x_r exp(-2 pi i k.(r - n//2)/n) / sqrt(N)``.
Everything here runs in float64 / complex128 unless a dtype is given.
"""

from __future__ import annotations

import math
from typing import Sequence

import numpy as np

OVERSAMP = 1.25
WIDTH = 4


def kb_beta(width: int = WIDTH, oversamp: float = OVERSAMP) -> float:
    """Kaiser-Bessel shape parameter (Beatty, Nishimura, Pauly 2005)."""
    return math.pi * math.sqrt((width / oversamp * (oversamp - 0.5)) ** 2 - 0.8)


def oversampled_shape(shape: Sequence[int], oversamp: float = OVERSAMP) -> tuple[int, ...]:
    return tuple(int(math.ceil(oversamp * int(n))) for n in shape)


def bessel_i0_as(x: np.ndarray) -> np.ndarray:
    """Modified Bessel I0 via Abramowitz & Stegun 9.8.1 (x < 3.75) and 9.8.2."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = x < 3.75
    t = x[small] / 3.75
    t2 = t * t
    out[small] = 1.0 + t2 * (3.5156229 + t2 * (3.0899424 + t2 * (1.2067492 + t2 * (
        0.2659732 + t2 * (0.0360768 + t2 * 0.0045813)))))
    xl = x[~small]
    u = 3.75 / xl
    poly = 0.39894228 + u * (0.01328592 + u * (0.00225319 + u * (-0.00157565 + u * (
        0.00916281 + u * (-0.02057706 + u * (0.02635537 + u * (-0.01647633 + u * 0.00392377)))))))
    out[~small] = np.exp(xl) / np.sqrt(xl) * poly
    return out


def kb_window(d: np.ndarray, beta: float) -> np.ndarray:
    """KB window at normalised distance d = (tap - k)/(w/2); zero for |d| > 1."""
    d = np.asarray(d, dtype=np.float64)
    inside = np.abs(d) <= 1.0
    arg = beta * np.sqrt(np.clip(1.0 - d * d, 0.0, None))
    return np.where(inside, bessel_i0_as(arg), 0.0)


def apodization_1d(n: int, os_n: int, width: int, beta: float) -> np.ndarray:
    """Per-axis de-apodisation a(i) = r/sinh(r) used on both sides of the NUFFT."""
    i = np.arange(n, dtype=np.float64)
    r = np.sqrt(beta * beta - (math.pi * width * (i - n // 2) / os_n) ** 2)
    return r / np.sinh(r)


def scale_coords(coord: np.ndarray, shape: Sequence[int], oversamp: float = OVERSAMP) -> np.ndarray:
    """Map grid-unit coordinates (..., 3) zyx onto the oversampled grid.

    Computed in float32 like the reference's float32 coordinate arrays.
    """
    c = np.array(coord, dtype=np.float32, copy=True)
    for ax in range(-len(shape), 0):
        n = int(shape[ax])
        os_n = int(math.ceil(oversamp * n))
        c[..., ax] *= np.float32(os_n / n)
        c[..., ax] += np.float32(os_n // 2)
    return c


def resize_center(x: np.ndarray, oshape: Sequence[int]) -> np.ndarray:
    """Centred zero-pad / crop over the trailing len(oshape) axes."""
    nd = len(oshape)
    ishape = x.shape[-nd:]
    out = np.zeros(x.shape[:-nd] + tuple(oshape), dtype=x.dtype)
    src, dst = [], []
    for i, o in zip(ishape, oshape):
        si = max(i // 2 - o // 2, 0)
        so = max(o // 2 - i // 2, 0)
        c = min(i - si, o - so)
        src.append(slice(si, si + c))
        dst.append(slice(so, so + c))
    lead = (slice(None),) * (x.ndim - nd)
    out[lead + tuple(dst)] = x[lead + tuple(src)]
    return out


def fftc(x: np.ndarray, axes=(-3, -2, -1)) -> np.ndarray:
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x, axes=axes), axes=axes), axes=axes)


def ifftc_unnorm(x: np.ndarray, axes=(-3, -2, -1)) -> np.ndarray:
    n = np.prod([x.shape[a] for a in axes])
    return np.fft.fftshift(np.fft.ifftn(np.fft.ifftshift(x, axes=axes), axes=axes), axes=axes) * n


def _tap_weights(ks: np.ndarray, width: int, beta: float):
    """Per-axis candidate taps (M, w+1) and their KB weights."""
    first = np.ceil(ks - width / 2.0).astype(np.int64)
    taps = first[:, None] + np.arange(width + 1, dtype=np.int64)[None, :]
    w = kb_window((taps - ks.astype(np.float64)[:, None]) / (width / 2.0), beta)
    return taps, w


def interpolate(grid: np.ndarray, ks: np.ndarray, width: int = WIDTH, beta: float | None = None) -> np.ndarray:
    """KB interpolation of grid (..., Gz, Gy, Gx) at scaled coords ks (M, 3) zyx."""
    beta = kb_beta(width) if beta is None else beta
    gshape = grid.shape[-3:]
    batch = grid.shape[:-3]
    g = grid.reshape((-1,) + gshape)
    ks = np.asarray(ks).reshape(-1, 3)
    tz, wz = _tap_weights(ks[:, 0], width, beta)
    ty, wy = _tap_weights(ks[:, 1], width, beta)
    tx, wx = _tap_weights(ks[:, 2], width, beta)
    tz %= gshape[0]
    ty %= gshape[1]
    tx %= gshape[2]
    out = np.zeros((g.shape[0], ks.shape[0]), dtype=np.result_type(grid.dtype, np.complex128))
    flat = g.reshape(g.shape[0], -1)
    nt = width + 1
    for a in range(nt):
        for b in range(nt):
            wzy = wz[:, a] * wy[:, b]
            base = (tz[:, a] * gshape[1] + ty[:, b]) * gshape[2]
            for c in range(nt):
                w = wzy * wx[:, c]
                idx = base + tx[:, c]
                out += w[None, :] * flat[:, idx]
    return out.reshape(batch + (ks.shape[0],))


def gridding(values: np.ndarray, ks: np.ndarray, gshape: Sequence[int], width: int = WIDTH,
             beta: float | None = None) -> np.ndarray:
    """Adjoint of ``interpolate``: spread values (..., M) onto grid (..., *gshape)."""
    beta = kb_beta(width) if beta is None else beta
    gshape = tuple(int(v) for v in gshape)
    batch = values.shape[:-1]
    v = values.reshape(-1, values.shape[-1]).astype(np.complex128)
    ks = np.asarray(ks).reshape(-1, 3)
    tz, wz = _tap_weights(ks[:, 0], width, beta)
    ty, wy = _tap_weights(ks[:, 1], width, beta)
    tx, wx = _tap_weights(ks[:, 2], width, beta)
    tz %= gshape[0]
    ty %= gshape[1]
    tx %= gshape[2]
    G = gshape[0] * gshape[1] * gshape[2]
    out = np.zeros((v.shape[0], G), dtype=np.complex128)
    nt = width + 1
    for a in range(nt):
        for b in range(nt):
            wzy = wz[:, a] * wy[:, b]
            base = (tz[:, a] * gshape[1] + ty[:, b]) * gshape[2]
            for c in range(nt):
                w = wzy * wx[:, c]
                idx = base + tx[:, c]
                for j in range(v.shape[0]):
                    contrib = w * v[j]
                    out[j] += np.bincount(idx, weights=contrib.real, minlength=G)
                    out[j] += 1j * np.bincount(idx, weights=contrib.imag, minlength=G)
    return out.reshape(batch + gshape)


def _apod_nd(shape: Sequence[int], oversamp: float, width: int, beta: float) -> np.ndarray:
    a = None
    for ax, n in enumerate(shape):
        os_n = int(math.ceil(oversamp * n))
        v = apodization_1d(n, os_n, width, beta)
        sh = [1] * len(shape)
        sh[ax] = n
        a = v.reshape(sh) if a is None else a * v.reshape(sh)
    return a


def nufft(image: np.ndarray, coord: np.ndarray, oversamp: float = OVERSAMP, width: int = WIDTH) -> np.ndarray:
    """Type-2 NUFFT of image (..., Z, Y, X) at coord (..., 3) zyx grid units.

    Restates SigPy 0.1.27 ``sigpy.nufft`` (called at ``nufft_backend.py:104-107``).
    Returns shape image.shape[:-3] + coord.shape[:-1], complex128.
    """
    beta = kb_beta(width, oversamp)
    shape = image.shape[-3:]
    os_shape = oversampled_shape(shape, oversamp)
    x = np.asarray(image, dtype=np.complex128) * _apod_nd(shape, oversamp, width, beta)
    x = x / math.sqrt(float(np.prod(shape)))
    x = resize_center(x, os_shape)
    grid = fftc(x)
    ks = scale_coords(coord, shape, oversamp)
    out = interpolate(grid, ks.reshape(-1, 3), width, beta) / width ** 3
    return out.reshape(image.shape[:-3] + coord.shape[:-1])


def nufft_adjoint(ksp: np.ndarray, coord: np.ndarray, oshape: Sequence[int], oversamp: float = OVERSAMP,
                  width: int = WIDTH) -> np.ndarray:
    """Type-1 adjoint NUFFT; restates SigPy 0.1.27 ``sigpy.nufft_adjoint``
    (called at ``nufft_backend.py:112-116`` with ``oshape=img_shape``)."""
    beta = kb_beta(width, oversamp)
    shape = tuple(int(v) for v in oshape[-3:])
    os_shape = oversampled_shape(shape, oversamp)
    npts = int(np.prod(coord.shape[:-1]))
    batch = ksp.shape[:ksp.ndim - (coord.ndim - 1)]
    vals = np.asarray(ksp, dtype=np.complex128).reshape(batch + (npts,))
    ks = scale_coords(coord, shape, oversamp).reshape(-1, 3)
    grid = gridding(vals, ks, os_shape, width, beta) / width ** 3
    x = ifftc_unnorm(grid)
    x = resize_center(x, shape)
    x = x / math.sqrt(float(np.prod(shape)))
    return x * _apod_nd(shape, oversamp, width, beta)


def nudft(image: np.ndarray, coord: np.ndarray) -> np.ndarray:
    """FP64 direct NUDFT y_j = N^{-1/2} sum_r x_r exp(-2 pi i k_j.(r - n//2)/n)."""
    shape = image.shape[-3:]
    N = float(np.prod(shape))
    k = np.asarray(coord, dtype=np.float64).reshape(-1, 3)
    x = np.asarray(image, dtype=np.complex128).reshape(image.shape[:-3] + (-1,))
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) - n // 2 for n in shape], indexing="ij")
    r = np.stack([g.ravel() / n for g, n in zip(grids, shape)], axis=1)  # (N, 3) in cycles
    out = np.empty(image.shape[:-3] + (k.shape[0],), dtype=np.complex128)
    chunk = max(1, int(2e7 // max(1, r.shape[0])))
    for s in range(0, k.shape[0], chunk):
        ph = np.exp(-2j * np.pi * (k[s:s + chunk] @ r.T))  # (m, N)
        out[..., s:s + chunk] = x @ ph.T
    return (out / math.sqrt(N)).reshape(image.shape[:-3] + coord.shape[:-1])


def nudft_adjoint(ksp: np.ndarray, coord: np.ndarray, oshape: Sequence[int]) -> np.ndarray:
    """FP64 direct adjoint of ``nudft``."""
    shape = tuple(int(v) for v in oshape[-3:])
    N = float(np.prod(shape))
    k = np.asarray(coord, dtype=np.float64).reshape(-1, 3)
    npts = k.shape[0]
    batch = ksp.shape[:ksp.ndim - (coord.ndim - 1)]
    y = np.asarray(ksp, dtype=np.complex128).reshape(batch + (npts,))
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) - n // 2 for n in shape], indexing="ij")
    r = np.stack([g.ravel() / n for g, n in zip(grids, shape)], axis=1)
    out = np.zeros(batch + (r.shape[0],), dtype=np.complex128)
    chunk = max(1, int(2e7 // max(1, r.shape[0])))
    for s in range(0, npts, chunk):
        ph = np.exp(2j * np.pi * (k[s:s + chunk] @ r.T))  # (m, N)
        out += y[..., s:s + chunk] @ ph
    return (out / math.sqrt(N)).reshape(batch + shape)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 error ||a - b|| / ||b|| in float64."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
