"""The allocation-free tolerance entry point against tr_pdhg_run's own tolerance.

tr_tolerance_sums_noalloc exists for callers that cannot allocate device
memory where they run the stopping test: hosts that own the whole device heap
through their own allocator and forbid a library from calling cudaMalloc.  It
keeps its partial sums in a fixed file-scope device array instead of
allocating.  Here it is called
through the C ABI on two consecutive PDHG iterates, and the tolerance it yields
must equal the one tr_pdhg_run reported for the same iteration.  This file is
named to be collected last, and it passes alone or after the other tests.
"""

import ctypes
import math

import numpy as np
import pytest

from _fixtures import binned, load_golden, pkg

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _solver(name):
    solver = pkg("solver")
    fx = load_golden(name)
    coords, dcfs, ksps = binned(fx)
    lam = float(fx["lam"])
    return solver.PdhgSolver(str(fx["alg"]), tuple(int(v) for v in fx["shape"]), coords, dcfs, fx["mps"], ksps,
                             l2_coupling=bool(fx["l2"]), lam_m=lam, lam_e=lam, lam_w1=lam, lam_w2=lam)


@pytest.mark.parametrize("name", ["tvme", "tvmw"])
def test_noalloc_tolerance_equals_pdhg_run_tolerance(name):
    torch = _torch()
    lib = pkg("_lib")
    L = lib.load()
    s = _solver(name)
    s.reset()
    sums = torch.zeros(2, dtype=torch.float64, device=s.device)   # caller-owned output
    alg = lib.TR_ALG[s.algorithm]
    for call in range(2):                                          # two calls in a row
        watched = s.u_bar if s.algorithm == "tvmw" else s.u
        prev = watched.clone()
        iters, tols = s.iterate(1, tol=0.0)
        assert iters == 1
        stream = torch.cuda.current_stream(s.device)
        st = L.tr_tolerance_sums_noalloc(ctypes.c_void_p(watched.data_ptr()), ctypes.c_void_p(prev.data_ptr()),
                                         watched.numel(), alg, ctypes.c_void_p(sums.data_ptr()),
                                         ctypes.c_void_p(stream.cuda_stream))
        lib.check(st, "tr_tolerance_sums_noalloc")
        num, den = sums.cpu().tolist()
        tol = math.sqrt(num) / (max(math.sqrt(den), 1e-12) if s.algorithm == "tvmw" else math.sqrt(den))
        assert math.isfinite(tol)
        assert abs(tol - tols[0]) <= 1e-9 * max(abs(tols[0]), 1e-30), (call, tol, tols[0])
    s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = _torch()
    lib = pkg("_lib")
    L = lib.load()
    x = torch.zeros(4, dtype=torch.complex64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    too_many = (64 * 1024 * 1024) + 1
    st = L.tr_tolerance_sums_noalloc(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), too_many,
                                     lib.TR_ALG["tvme"], ctypes.c_void_p(out.data_ptr()), None)
    assert st == lib.TR_ERR_INVALID_ARG
    assert "exceeds the maximum" in lib.last_error()
