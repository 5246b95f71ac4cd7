"""Shared helpers for the test-suite (loading golden fixtures, building problems)."""

from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

PKG_NAME = "multinodemri-miccai26_b200"


def pkg(sub: str | None = None):
    return importlib.import_module(PKG_NAME if sub is None else f"{PKG_NAME}.{sub}")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"pdhg_{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def binned(fx: dict):
    """Split a fixture into per-bin coords, dcf and k-space with the reference's rule."""
    edges = fx["bin_edges"]
    resp = fx["resp"]
    coords, dcfs, ksps = [], [], []
    for b in range(len(edges) - 1):
        idx = (resp >= edges[b]) & (resp < edges[b + 1])
        coords.append(fx["coord"][idx])
        dcfs.append(fx["dcf"][idx])
        ksps.append(fx["ksp"][:, :, idx])
    return coords, dcfs, ksps


def oracle_problem(fx: dict, dtype=np.complex128):
    from oracle import pdhg as op
    coords, dcfs, ksps = binned(fx)
    shape = tuple(int(v) for v in fx["shape"])
    nf = op.OracleNufft(shape, coords, out_dtype=dtype)
    return op.Problem(nufft=nf, ksp=[k.astype(dtype) for k in ksps], dcf=dcfs, mps=fx["mps"], dtype=dtype)
