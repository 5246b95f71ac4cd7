"""CPU-side checks of the C ABI library: it builds, loads and exports the header's symbols."""

import ctypes
import re
import subprocess
import sys

import pytest

from _fixtures import REPO, pkg

HEADER = REPO / "include" / "toporecon_b200.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:tr_status|const char\*)\s+(tr_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("tr_plan_create", "tr_plan_destroy", "tr_nufft_forward", "tr_nufft_adjoint", "tr_pdhg_run",
                 "tr_last_error_string"):
        assert must in names


def test_library_loads_and_exports_every_declared_symbol():
    build = pkg("build")
    lib_path = build.build()
    lib = ctypes.CDLL(str(lib_path))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_signatures_cover_header():
    lib_mod = pkg("_lib")
    assert set(declared_functions()) <= set(lib_mod.EXPORTED)


def test_error_string_without_gpu():
    lib = pkg("_lib").load()
    # tr_plan_create with a null descriptor fails cleanly (no GPU needed)
    handle = ctypes.c_void_p()
    st = lib.tr_plan_create(None, ctypes.byref(handle))
    assert st == pkg("_lib").TR_ERR_INVALID_ARG
    assert "null" in pkg("_lib").last_error()


def test_registry_rejects_unknown_backend():
    nb = pkg("nufft_backend")
    with pytest.raises(ValueError, match="Unknown NUFFT backend"):
        nb.create_nufft_backend("cufinufft", img_shape=(8, 8, 8), coordinates=[], device=0)


def test_abc_validates_shape_and_bins():
    nb = pkg("nufft_backend")

    class Dummy(nb.NufftBackend):
        xp = None
        num_bins = 2

        def to_device(self, a):
            return a

        def forward(self, image, bin_index):
            return self._validate_bin(bin_index)

        def adjoint(self, k, bin_index):
            return self._validate_bin(bin_index)

    with pytest.raises(ValueError):
        Dummy((8, 8))
    d = Dummy((8, 8, 8))
    assert d.forward(None, 1) == 1
    with pytest.raises(IndexError):
        d.forward(None, 2)


def test_sigpy_backend_reports_missing_dependency():
    nb = pkg("nufft_backend")
    try:
        import sigpy  # noqa: F401
        import toporecon.nufft_backend  # noqa: F401
        pytest.skip("the reference package and SigPy are installed")
    except ImportError:
        pass
    with pytest.raises(RuntimeError, match="cannot be imported here"):
        nb.create_nufft_backend("sigpy", img_shape=(8, 8, 8), coordinates=[[[0.0, 0.0, 0.0]]], device=-1)
    with pytest.raises(ValueError, match="Unknown NUFFT backend"):
        nb.create_nufft_backend("cufinufft", img_shape=(8, 8, 8), coordinates=[[[0.0, 0.0, 0.0]]], device=0)
