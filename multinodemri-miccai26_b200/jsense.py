"""JSENSE coil-sensitivity estimation on the b200 NUFFT.

Same entry point as the reference's ``estimate_sensitivity_maps``
(``preprocessing/jsense.py:33-98``): first echo only, maps estimated on a
calibration grid and resized per coil in the Fourier domain to the image grid.
The reference delegates the estimation to SigPy's ``JsenseRecon``; this module
restates the published JSENSE method (joint image and sensitivity estimation,
Ying & Sheng 2007) with SigPy's application defaults:

* calibration samples: every |k_i| < calibration width / 2, on a
  width^3 grid; k-space divided by its largest magnitude;
* unknowns: the image x (start: ones) and per-coil kernels K_c of
  kernel-width^3 Fourier coefficients (start: zeros), maps S_c = IFFT(pad(K_c));
* alternating minimisation of sum_c ||w^(1/2) (F(S_c x) - y_c)||^2 + lambda (...):
  kernels with x fixed, then x with the maps fixed, each by ``max_inner_iter``
  conjugate-gradient steps on the normal equations, warm-started.

Every NUFFT runs through two b200 plans on the calibration trajectory (one with
the coils as coil maps for the image step, one with the coils as separate
images for the kernel step), with the density weights applied in the
deterministic gridding; the small centred FFTs of the map parameterisation and
the CG vector algebra are torch on the same device.  The oracle is
``oracle/jsense.py``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Optional, Sequence

import numpy as np


@dataclass(frozen=True)
class JsenseConfig:
    """The reference's JSENSE settings (``preprocessing/jsense.py:16-30``); ``None``
    keeps the SigPy application defaults (16, 24, 0, 10, 10)."""

    readout_fraction: float = 0.95
    coordinate_scaling: str = "legacy_max"
    mps_kernel_width: Optional[int] = None
    kspace_calibration_width: Optional[int] = None
    regularization: Optional[float] = None
    max_iter: Optional[int] = None
    max_inner_iter: Optional[int] = None


def _fft_ortho(torch, x):
    dims = (-3, -2, -1)
    return torch.fft.fftshift(torch.fft.fftn(torch.fft.ifftshift(x, dim=dims), dim=dims, norm="ortho"), dim=dims)


def _ifft_ortho(torch, x):
    dims = (-3, -2, -1)
    return torch.fft.fftshift(torch.fft.ifftn(torch.fft.ifftshift(x, dim=dims), dim=dims, norm="ortho"), dim=dims)


def _resize(torch, x, shape):
    """Centred zero-pad / crop of the last three axes (the NUFFT's convention)."""
    out = torch.zeros(x.shape[:-3] + tuple(shape), dtype=x.dtype, device=x.device)
    src, dst = [], []
    for i, o in zip(x.shape[-3:], shape):
        si, so = max(i // 2 - o // 2, 0), max(o // 2 - i // 2, 0)
        c = min(i - si, o - so)
        src.append(slice(si, si + c))
        dst.append(slice(so, so + c))
    out[(...,) + tuple(dst)] = x[(...,) + tuple(src)]
    return out


def _cg(torch, normal, rhs, x0, iters):
    x = x0.clone()
    r = rhs - normal(x)
    p = r.clone()
    rr = float(torch.vdot(r.reshape(-1), r.reshape(-1)).real)
    for _ in range(iters):
        if rr == 0.0:
            break
        ap = normal(p)
        alpha = rr / float(torch.vdot(p.reshape(-1), ap.reshape(-1)).real)
        x = x + alpha * p
        r = r - alpha * ap
        rr_new = float(torch.vdot(r.reshape(-1), r.reshape(-1)).real)
        p = r + (rr_new / rr) * p
        rr = rr_new
    return x


def jsense_calibration(y, coord, weights, *, device=0, ker_width: int = 16, calib_width: int = 24,
                       lamda: float = 0.0, max_iter: int = 10, inner: int = 10):
    """Maps (C, w, w, w) on the calibration grid, torch complex64 on ``device``,
    from (C, M) k-space, (M, 3) zyx grid-unit coordinates and (M,) weights."""
    import torch
    from .nufft_backend import B200NufftBackend
    y = np.asarray(y)
    coord = np.asarray(coord, np.float32).reshape(-1, 3)
    weights = np.asarray(weights, np.float32).reshape(-1)
    keep = np.all(np.abs(coord) < calib_width / 2.0, axis=-1)
    if not np.any(keep):
        raise ValueError("no k-space samples inside the calibration region")
    yc, kc, wc = y[:, keep], coord[keep], weights[keep]
    C = yc.shape[0]
    shape = (calib_width,) * 3
    kshape = (ker_width,) * 3
    # image step: coils as coil maps of one image; kernel step: coils as C images under unit maps
    px = B200NufftBackend(shape, [kc], device, dcf=[wc], n_coils=C, n_echoes=1)
    pk = B200NufftBackend(shape, [kc], device, dcf=[wc], n_coils=1, n_echoes=C)
    dev = px.device
    try:
        pk.set_maps(torch.ones((1,) + shape, dtype=torch.complex64, device=dev))
        ys = torch.from_numpy(np.ascontiguousarray(yc.astype(np.complex64))).to(dev)
        scale = float(ys.abs().max())
        ys = ys / (scale if scale > 0 else 1.0)
        yint = px.sort_kspace(ys, 0)                       # (M, C) tile-sorted; same order in both plans
        x = torch.ones(shape, dtype=torch.complex64, device=dev)
        K = torch.zeros((C,) + kshape, dtype=torch.complex64, device=dev)
        for _ in range(max_iter):
            xs = x

            def AKhAK(k):
                imgs = _ifft_ortho(torch, _resize(torch, k, shape)) * xs
                r = pk.forward_bin(imgs, 0)
                return _resize(torch, _fft_ortho(torch, torch.conj(xs) * pk.adjoint_bin(r, 0, use_dcf=True)),
                               kshape) + lamda * k

            rhs_k = _resize(torch, _fft_ortho(torch, torch.conj(xs) * pk.adjoint_bin(yint, 0, use_dcf=True)), kshape)
            K = _cg(torch, AKhAK, rhs_k, K, inner)
            px.set_maps(_ifft_ortho(torch, _resize(torch, K, shape)))

            def AxhAx(im):
                return px.adjoint_bin(px.forward_bin(im[None], 0), 0, use_dcf=True)[0] + lamda * im

            rhs_x = px.adjoint_bin(yint, 0, use_dcf=True)[0]
            x = _cg(torch, AxhAx, rhs_x, x, inner)
        maps = _ifft_ortho(torch, _resize(torch, K, shape))
        torch.cuda.synchronize(dev)
        return maps
    finally:
        px.close()
        pk.close()


def resize_maps(maps, image_shape: Sequence[int]):
    """Per-coil Fourier-domain resize to the image grid (``preprocessing/jsense.py:93-96``)."""
    import torch
    return _ifft_ortho(torch, _resize(torch, _fft_ortho(torch, maps), tuple(int(v) for v in image_shape)))


def estimate_sensitivity_maps(kspace, coordinates_zyx, density, *, image_shape_zyx: Sequence[int],
                              device: Any = 0, show_progress: bool = False,
                              config: Optional[JsenseConfig] = None) -> np.ndarray:
    """``[coil, z, y, x]`` complex64 maps from ``[echo, coil, trajectory, readout]``
    k-space (first echo), ``[trajectory, readout, 3]`` zyx coordinates and
    ``[trajectory, readout]`` density: the reference's entry point and checks."""
    data = np.asarray(kspace)
    if data.ndim != 4:
        raise ValueError(f"k-space must have shape [echo,coil,trajectory,readout], got {data.shape}.")
    coordinates = np.asarray(coordinates_zyx)
    weights = np.asarray(density)
    if coordinates.shape[:-1] != data.shape[-2:]:
        raise ValueError(f"trajectory shape {coordinates.shape} does not match k-space {data.shape[-2:]}.")
    if weights.shape != data.shape[-2:]:
        raise ValueError(f"density shape {weights.shape} does not match k-space {data.shape[-2:]}.")
    cfg = config or JsenseConfig()
    maps = jsense_calibration(
        data[0].reshape(data.shape[1], -1), coordinates.reshape(-1, 3), weights.reshape(-1), device=device,
        ker_width=cfg.mps_kernel_width or 16, calib_width=cfg.kspace_calibration_width or 24,
        lamda=cfg.regularization or 0.0, max_iter=cfg.max_iter or 10, inner=cfg.max_inner_iter or 10)
    return resize_maps(maps, image_shape_zyx).cpu().numpy().astype(np.complex64)
