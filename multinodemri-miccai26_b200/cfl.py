"""BART-style CFL/HDR arrays in the reference's convention (single-rank I/O for the CLI).

The reference stores the payload in C order while listing the dimensions in
reverse in the ``.hdr`` file (``src/toporecon/data/cfl.py:14-115``); the
k-space file is nine-dimensional ``(1, 1, 1, E, 1, C, TR, RO, 1)``
(``data/dataset.py:54-88``).  Only what the b200 CLI needs is provided:
read / write whole arrays, read the header, memory-map the payload.
"""

from __future__ import annotations

from pathlib import Path
from typing import Sequence

import numpy as np

CFL_DTYPE = np.dtype(np.complex64)


def base_path(name) -> Path:
    p = Path(name)
    return p.with_suffix("") if p.suffix in (".cfl", ".hdr") else p


def read_header(name) -> tuple:
    path = base_path(name).with_suffix(".hdr")
    with path.open("r", encoding="utf-8") as fh:
        for line in fh:
            s = line.strip()
            if s and not s.startswith("#"):
                dims = [int(v) for v in s.split()]
                if any(d < 1 for d in dims):
                    raise ValueError(f"{path}: every CFL dimension has to be at least 1, header lists {dims}")
                return tuple(reversed(dims))
    raise ValueError(f"{path}: the header holds no dimension line")


def read(name, mmap: bool = False) -> np.ndarray:
    root = base_path(name)
    shape = read_header(root)
    payload = root.with_suffix(".cfl")
    expected = int(np.prod(shape, dtype=np.int64)) * CFL_DTYPE.itemsize
    if payload.stat().st_size != expected:
        raise ValueError(f"{payload}: holds {payload.stat().st_size} bytes, but the header's shape "
                         f"{shape} needs {expected}")
    if mmap:
        return np.memmap(payload, mode="r", dtype=CFL_DTYPE, shape=shape)
    return np.fromfile(payload, dtype=CFL_DTYPE).reshape(shape)


def write(name, array: np.ndarray) -> None:
    root = base_path(name)
    root.parent.mkdir(parents=True, exist_ok=True)
    arr = np.ascontiguousarray(np.asarray(array, dtype=CFL_DTYPE))
    with root.with_suffix(".hdr").open("w", encoding="utf-8") as fh:
        fh.write("# Dimensions\n")
        fh.write(" ".join(str(d) for d in reversed(arr.shape)) + "\n")
    arr.tofile(root.with_suffix(".cfl"))


def kspace_layout(shape: Sequence[int]) -> tuple:
    """(echoes, coils, trajectories, readout) of the nine-dimensional k-space file."""
    dims = tuple(int(v) for v in shape)
    if len(dims) < 8:
        raise ValueError(f"k-space CFL must contain at least eight dimensions; found {dims}.")
    E, C, TR, RO = dims[-6], dims[-4], dims[-3], dims[-2]
    if E * C * TR * RO != int(np.prod(dims, dtype=np.int64)):
        raise ValueError(f"Unsupported non-singleton dimensions in k-space CFL shape {dims}.")
    return E, C, TR, RO


def read_kspace(name, echo_start: int, echo_end: int, readout: int, trajectory_indices: np.ndarray) -> np.ndarray:
    """(E_local, C, N_tr, readout) complex64 selected from the memory-mapped file."""
    mm = read(name, mmap=True)
    E, C, TR, RO = kspace_layout(mm.shape)
    view = mm.reshape(E, C, TR, RO)
    idx = np.asarray(trajectory_indices, dtype=np.int64)
    return np.ascontiguousarray(view[echo_start:echo_end][:, :, idx, :readout])


def read_maps(name) -> np.ndarray:
    """(C, Z, Y, X) complex64 coil maps from a (..., C, Z, Y, X)-trailing CFL."""
    arr = read(name)
    squeezed = arr.reshape((-1,) + arr.shape[-3:])
    return np.ascontiguousarray(squeezed)
