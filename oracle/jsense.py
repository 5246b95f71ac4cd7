"""JSENSE coil-sensitivity estimation, CPU restatement (TEST INFRASTRUCTURE ONLY).

The reference calls SigPy 0.1.27's ``mr.app.JsenseRecon`` on the first echo
(``preprocessing/jsense.py:33-98``), then resizes every map to the image grid
in the Fourier domain (``:93-96``).  SigPy is not available here, so this file
restates the published JSENSE method (joint image and sensitivity estimation,
Ying & Sheng 2007) with SigPy's application defaults (kernel width 16,
calibration width 24, lambda 0, 10 outer and 10 inner iterations):

* calibration data: samples with every |k_i| < calib_width / 2, on a
  calib_width^3 grid, k-space divided by its largest magnitude;
* unknowns: image x (init ones) and per-coil kernels K_c of ker_width^3
  Fourier coefficients (init zeros); maps S_c = IFFT(zero-pad(K_c));
* alternating minimisation of sum_c ||w^(1/2) (F(S_c x) - y_c)||^2 + lambda (...):
  first the kernels with x fixed, then x with the maps fixed, each by
  ``inner`` conjugate-gradient steps on the normal equations, warm-started;
* output: the maps on the calibration grid.

Parity with SigPy is unpinned (no SigPy here); this is the oracle of the b200
JSENSE (``multinodemri-miccai26_b200/jsense.py``), which must match it.
Complex128 throughout.
"""

from __future__ import annotations

import math

import numpy as np

from . import nufft as onf


def fft_ortho(x):
    n = np.prod(x.shape[-3:])
    return onf.fftc(x) / math.sqrt(n)


def ifft_ortho(x):
    n = np.prod(x.shape[-3:])
    return onf.ifftc_unnorm(x) / math.sqrt(n)


def calibration(y, coord, weights, calib_width):
    """(C, M) k-space, (M, 3) coordinates, (M,) weights -> the calibration subset."""
    keep = np.all(np.abs(coord) < calib_width / 2.0, axis=-1)
    return y[:, keep], coord[keep], weights[keep]


def cg(normal, rhs, x0, iters):
    """Conjugate gradients on a Hermitian positive semi-definite normal operator."""
    x = x0.copy()
    r = rhs - normal(x)
    p = r.copy()
    rr = np.vdot(r, r).real
    for _ in range(iters):
        if rr == 0.0:
            break
        ap = normal(p)
        alpha = rr / np.vdot(p, ap).real
        x = x + alpha * p
        r = r - alpha * ap
        rr_new = np.vdot(r, r).real
        p = r + (rr_new / rr) * p
        rr = rr_new
    return x


def jsense(y, coord, weights, ker_width=16, calib_width=24, lamda=0.0, max_iter=10, inner=10, nufft=None,
           nufft_adjoint=None):
    """Maps (C, w, w, w) on the calibration grid from (C, M) k-space.  ``nufft`` /
    ``nufft_adjoint`` default to the restatement in ``oracle/nufft.py``; the timed
    CPU baseline passes the C/OpenMP loops of ``oracle/cgrid.py``."""
    y, coord, w = calibration(np.asarray(y, np.complex128), np.asarray(coord, np.float64),
                              np.asarray(weights, np.float64), calib_width)
    shape = (calib_width,) * 3
    C = y.shape[0]
    scale = np.max(np.abs(y)) if y.size else 1.0
    y = y / (scale if scale > 0 else 1.0)
    fwd = nufft or onf.nufft
    adj = nufft_adjoint or onf.nufft_adjoint
    F = lambda im: fwd(im, coord)                                        # (..., Z, Y, X) -> (..., M)
    FH = lambda k: adj(k, coord, shape)
    pad = lambda k: onf.resize_center(k, shape)
    crop = lambda im: onf.resize_center(im, (ker_width,) * 3)
    x = np.ones(shape, np.complex128)
    K = np.zeros((C,) + (ker_width,) * 3, np.complex128)
    for _ in range(max_iter):
        xs = x
        AK = lambda k: F(ifft_ortho(pad(k)) * xs)
        AKH = lambda r: crop(fft_ortho(np.conj(xs) * FH(r)))
        K = cg(lambda k: AKH(w * AK(k)) + lamda * k, AKH(w * y), K, inner)
        S = ifft_ortho(pad(K))
        Ax = lambda im: F(S * im)
        AxH = lambda r: np.sum(np.conj(S) * FH(r), axis=0)
        x = cg(lambda im: AxH(w * Ax(im)) + lamda * im, AxH(w * y), x, inner)
    return ifft_ortho(pad(K))


def resize_maps(maps, image_shape):
    """The reference's per-coil Fourier-domain resize to the image grid
    (``preprocessing/jsense.py:93-96``: ifft(resize(fft(map), shape)))."""
    return np.stack([ifft_ortho(onf.resize_center(fft_ortho(m), image_shape)) for m in maps])
