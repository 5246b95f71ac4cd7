"""Multi-threaded CPU NUFFT: the oracle restatement with C/OpenMP KB loops (test
infrastructure and the timed CPU baseline only).

``nufft`` / ``nufft_adjoint`` follow ``oracle.nufft`` exactly (SigPy 0.1.27
definition, reference call sites ``nufft_backend.py:104-116``) but run the
interpolation / gridding loops in ``kbgrid.c`` (OpenMP) and the FFTs in
``scipy.fft`` with every host thread, in complex64 like SigPy's CPU path.
``build()`` compiles ``libkbgrid.so`` next to this file with gcc.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np
import scipy.fft as sfft

from . import nufft as onf

HERE = Path(__file__).resolve().parent
SRC = HERE / "kbgrid.c"
LIB = HERE / "libkbgrid.so"
_lib = None


def threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run(["gcc", "-O3", "-fopenmp", "-shared", "-fPIC", "-o", str(tmp), str(SRC), "-lm"], check=True)
        os.replace(tmp, LIB)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        f32p = ctypes.POINTER(ctypes.c_float)
        lib.kb_interpolate.argtypes = [f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, f32p,
                                       ctypes.c_long, ctypes.c_int, ctypes.c_double, f32p]
        lib.kb_gridding.argtypes = [f32p, ctypes.c_int, f32p, ctypes.c_long, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, f32p, ctypes.c_int]
        _lib = lib
    return _lib


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def interpolate(grid: np.ndarray, ks: np.ndarray, width=onf.WIDTH, beta=None) -> np.ndarray:
    beta = onf.kb_beta(width) if beta is None else beta
    g = np.ascontiguousarray(grid, dtype=np.complex64)
    gshape = g.shape[-3:]
    batch = int(np.prod(g.shape[:-3])) if g.ndim > 3 else 1
    k = np.ascontiguousarray(ks, dtype=np.float32).reshape(-1, 3)
    out = np.empty((batch, k.shape[0]), dtype=np.complex64)
    load().kb_interpolate(_fp(g), batch, *gshape, _fp(k), k.shape[0], width, beta, _fp(out))
    return out.reshape(g.shape[:-3] + (k.shape[0],))


def gridding(vals: np.ndarray, ks: np.ndarray, gshape, width=onf.WIDTH, beta=None) -> np.ndarray:
    beta = onf.kb_beta(width) if beta is None else beta
    v = np.ascontiguousarray(vals, dtype=np.complex64)
    batch = int(np.prod(v.shape[:-1])) if v.ndim > 1 else 1
    k = np.ascontiguousarray(ks, dtype=np.float32).reshape(-1, 3)
    out = np.empty((batch,) + tuple(gshape), dtype=np.complex64)
    nslab = max(1, min(int(gshape[0]), 4 * threads()))
    load().kb_gridding(_fp(v), batch, _fp(k), k.shape[0], width, beta, *gshape, _fp(out), nslab)
    return out.reshape(v.shape[:-1] + tuple(gshape))


def nufft(image: np.ndarray, coord: np.ndarray, oversamp=onf.OVERSAMP, width=onf.WIDTH) -> np.ndarray:
    beta = onf.kb_beta(width, oversamp)
    shape = image.shape[-3:]
    os_shape = onf.oversampled_shape(shape, oversamp)
    x = (image * onf._apod_nd(shape, oversamp, width, beta).astype(np.float32)).astype(np.complex64)
    x /= np.float32(math.sqrt(float(np.prod(shape))))
    x = onf.resize_center(x, os_shape)
    ax = (-3, -2, -1)
    grid = sfft.fftshift(sfft.fftn(sfft.ifftshift(x, axes=ax), axes=ax, workers=threads()), axes=ax)
    ks = onf.scale_coords(coord, shape, oversamp).reshape(-1, 3)
    out = interpolate(grid, ks, width, beta) / np.float32(width ** 3)
    return out.reshape(image.shape[:-3] + coord.shape[:-1])


def nufft_adjoint(ksp: np.ndarray, coord: np.ndarray, oshape, oversamp=onf.OVERSAMP, width=onf.WIDTH) -> np.ndarray:
    beta = onf.kb_beta(width, oversamp)
    shape = tuple(int(v) for v in oshape[-3:])
    os_shape = onf.oversampled_shape(shape, oversamp)
    npts = int(np.prod(coord.shape[:-1]))
    batch = ksp.shape[:ksp.ndim - (coord.ndim - 1)]
    vals = np.asarray(ksp, dtype=np.complex64).reshape(batch + (npts,))
    ks = onf.scale_coords(coord, shape, oversamp).reshape(-1, 3)
    grid = gridding(vals, ks, os_shape, width, beta) / np.float32(width ** 3)
    ax = (-3, -2, -1)
    G = float(np.prod(os_shape))
    x = sfft.fftshift(sfft.ifftn(sfft.ifftshift(grid, axes=ax), axes=ax, workers=threads()), axes=ax)
    x = onf.resize_center(x, shape) * np.float32(G / math.sqrt(float(np.prod(shape))))
    return (x * onf._apod_nd(shape, oversamp, width, beta).astype(np.float32)).astype(np.complex64)
