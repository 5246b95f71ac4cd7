"""Generate golden PDHG vectors by running the reference's own reconstructors.

Run in the build container (where the reference source is mounted):

    python tests/golden/make_golden.py /path/to/reference

The reference's ``TvmReconstructor`` (``algorithms/tvm.py:63-491``),
``TvmeReconstructor`` (``algorithms/tvme.py:56-575``) and
``TvmwReconstructor`` (``algorithms/tvmw.py:213-786``) are imported from the
reference tree and run unmodified, single rank, on small seeded problems.
Their third-party dependencies are absent here and are replaced by shims:

* ``mpi4py``  -- a one-rank stand-in (``Request.Waitall`` over empty request
  lists); all halo peers are absent, so every ghost is a global edge;
* ``sigpy``   -- CPU device, ``to_device``, ``axpy`` and ``nufft`` /
  ``nufft_adjoint`` backed by ``oracle.nufft`` (the SigPy 0.1.27 restatement),
  returning complex64 like SigPy;
* ``ptwt``    -- ``wavedec3`` / ``waverec3`` backed by ``oracle.wavelets``;
* ``cupy``    -- an inert module (TVMW's DLPack helpers import it by name).

So the fixtures pin the reference's PDHG loop (update order, boundaries,
proximal maps, W1, the W2 usage pattern and the stopping rule) with the NUFFT
and db6 restatements inside; they do not pin SigPy or ptwt themselves.
Outputs: ``tests/golden/pdhg_<alg>.npz``.
"""

from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from oracle import nufft as onf  # noqa: E402
from oracle import wavelets as owv  # noqa: E402


# ----------------------------------------------------------------- shims
def _install_shims():
    mpi = types.ModuleType("mpi4py")
    MPI = types.SimpleNamespace()

    class _Request:
        @staticmethod
        def Waitall(reqs):
            assert not reqs
    MPI.Request = _Request
    MPI.Comm = object
    MPI.SUM = "sum"
    MPI.MAX = "max"
    MPI.IN_PLACE = None
    MPI.PROC_NULL = -2
    MPI.COMM_NULL = None
    MPI.REQUEST_NULL = None
    MPI.COMM_TYPE_SHARED = 0
    MPI.UNDEFINED = -32766
    MPI.TAG_UB = 0
    MPI.COMM_WORLD = None
    mpi.MPI = MPI
    sys.modules["mpi4py"] = mpi

    sp = types.ModuleType("sigpy")

    class Device:
        def __init__(self, dev=-1):
            self.id = getattr(dev, "id", dev)
            self.xp = np

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False
    sp.Device = Device
    sp.cpu_device = Device(-1)
    sp.to_device = lambda a, device=None: np.asarray(a)

    def axpy(y, a, x):
        y += a * x
    sp.axpy = axpy

    def nufft(x, coord, oversamp=1.25, width=4):
        assert oversamp == 1.25 and width == 4
        return onf.nufft(x, coord).astype(np.complex64)

    def nufft_adjoint(y, coord, oshape=None, oversamp=1.25, width=4):
        return onf.nufft_adjoint(y, coord, oshape).astype(np.complex64)
    sp.nufft = nufft
    sp.nufft_adjoint = nufft_adjoint
    sys.modules["sigpy"] = sp

    cp = types.ModuleType("cupy")

    class _NotCupy:  # no object is ever an instance
        pass
    cp.ndarray = _NotCupy
    cp.complex64 = np.complex64
    cp.float32 = np.float32
    cp.ascontiguousarray = np.ascontiguousarray
    cp.asarray = np.asarray
    cp.cuda = types.SimpleNamespace(get_current_stream=lambda: None)
    sys.modules["cupy"] = cp

    import torch

    # TVMW's DLPack helpers synchronise the CUDA device around every crossing
    # (tvmw.py:84-107, :200, :205); with CPU tensors that is a no-op.
    torch.cuda.synchronize = lambda device=None: None

    pt = types.ModuleType("ptwt")

    def wavedec3(t, wavelet, mode="zero", level=None, axes=(-3, -2, -1)):
        assert mode == "zero" and tuple(axes) == (-3, -2, -1)
        c = owv.wavedec3(t.detach().cpu().numpy().astype(np.float64), wavelet, level)
        conv = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32))
        return [conv(c[0])] + [{k: conv(v) for k, v in d.items()} for d in c[1:]]

    def waverec3(coeffs, wavelet, axes=(-3, -2, -1)):
        c = [coeffs[0].numpy().astype(np.float64)] + \
            [{k: v.numpy().astype(np.float64) for k, v in d.items()} for d in coeffs[1:]]
        return torch.from_numpy(np.ascontiguousarray(owv.waverec3(c, wavelet), dtype=np.float32))
    pt.wavedec3 = wavedec3
    pt.waverec3 = waverec3
    sys.modules["ptwt"] = pt


class FakeGrid:
    def halo_exchange(self, sendbuf, recvbuf, send_peer=None, recv_peer=None, tag=0):
        return []


def _tagger(it, axis="motion", kind="delta"):
    return 0


# ----------------------------------------------------------------- problems
def small_problem(shape, C, E, B, TR, RO, seed):
    sys.path.insert(0, str(REPO))
    import importlib
    syn = importlib.import_module("multinodemri-miccai26_b200.synthetic")
    cfg = syn.SyntheticConfig("golden", tuple(shape), C, E, B, TR, RO, seed=seed, n_ellipsoids=3)
    ds = syn.make_geometry(cfg)

    def fwd(imgs, coords):
        return onf.nufft(imgs, coords).astype(np.complex64)
    syn.simulate_kspace(ds, fwd)
    return ds


def run_reference(alg, ds, iters, tol, **kw):
    mod = __import__(f"toporecon.algorithms.{alg}", fromlist=["x"])
    cfg = ds.cfg
    edges = np.asarray(ds.meta["bin_edges"], dtype=np.float64)
    common = dict(max_iter=iters, tol=tol, margin=0, device=-1, B_total=cfg.n_bins, b0=0, b1=cfg.n_bins,
                  bin_edges=edges, dist_grid=FakeGrid(), tagger=_tagger, show_pbar=False,
                  nufft_backend="sigpy", sigma=1 / 6, tau=1 / 6)
    dual_q = np.zeros_like(ds.ksp)
    if alg == "tvm":
        rec = mod.TvmReconstructor(ds.ksp, ds.coord, ds.dcf, ds.mps, ds.resp, dual_q, cfg.n_bins,
                                   kw.get("l2", False), lamda=kw["lam"], **common)
    elif alg == "tvme":
        rec = mod.TvmeReconstructor(ds.ksp, ds.coord, ds.dcf, ds.mps, ds.resp, dual_q, cfg.n_bins,
                                    kw.get("l2", False), lamda_m=kw["lam"], lamda_e=kw["lam"],
                                    E_total=cfg.n_echoes, e0=0, e1=cfg.n_echoes, **common)
    else:
        rec = mod.TvmwReconstructor(ds.ksp, ds.coord, ds.dcf, ds.mps, ds.resp, dual_q, cfg.n_bins,
                                    kw.get("l2", False), lambda1=kw["lam"], lambda2=kw["lam"],
                                    lambda3=kw["lam"], E_total=cfg.n_echoes, e0=0, e1=cfg.n_echoes,
                                    **common)
    calls = {"n": 0}
    orig_pdhg = rec.pdhg

    def counted(*a):
        calls["n"] += 1
        return orig_pdhg(*a)
    rec.pdhg = counted
    out = rec.run()
    return np.asarray(out), calls["n"]


CASES = {
    # name: (alg, shape, C, E, B, TR, RO, seed, kwargs)
    "tvm": ("tvm", (12, 16, 16), 2, 1, 3, 48, 24, 11, dict(lam=1e-3)),
    "tvm_l2": ("tvm", (12, 16, 16), 2, 2, 3, 48, 24, 12, dict(lam=1e-3, l2=True)),
    "tvme": ("tvme", (12, 16, 16), 2, 3, 3, 48, 24, 13, dict(lam=1e-3)),
    "tvme_l2": ("tvme", (12, 16, 16), 2, 3, 2, 48, 24, 14, dict(lam=1e-3, l2=True)),
    "tvmw": ("tvmw", (24, 24, 22), 2, 3, 2, 64, 28, 15, dict(lam=1e-3)),
}


def main(ref_root: str):
    sys.path.insert(0, str(Path(ref_root) / "src"))
    _install_shims()
    for name, (alg, shape, C, E, B, TR, RO, seed, kw) in CASES.items():
        ds = small_problem(shape, C, E, B, TR, RO, seed)
        iters = 4
        img_k, _ = run_reference(alg, ds, iters, 0.0, **kw)
        img_tol, n_tol = run_reference(alg, ds, 60, 2e-2, **kw)
        np.savez_compressed(
            HERE / f"pdhg_{name}.npz",
            alg=alg, shape=np.array(shape), n_iter=iters, lam=kw["lam"], l2=bool(kw.get("l2", False)),
            coord=ds.coord, dcf=ds.dcf, resp=ds.resp, mps=ds.mps, ksp=ds.ksp,
            bin_edges=np.asarray(ds.meta["bin_edges"]), image_k=img_k.astype(np.complex64),
            tol_stop=2e-2, iters_tol=n_tol, image_tol=img_tol.astype(np.complex64))
        print(name, img_k.shape, float(np.abs(img_k).max()), "iters to tol", n_tol)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the reference source tree>")
    main(sys.argv[1])
