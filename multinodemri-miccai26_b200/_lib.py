"""ctypes binding of ``libtoporecon_b200.so`` (the C ABI in include/toporecon_b200.h).

The shared library is built in-tree by ``build.py`` and loaded from this
directory.  There is no fallback: if the library or a CUDA device is missing,
every entry point raises.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtoporecon_b200.so"

TR_OK = 0
TR_ERR_INVALID_ARG = 1
TR_ERR_OOM = 2
TR_ERR_NONFINITE = 3
TR_ERR_TIMEOUT = 4
TR_ERR_CUDA = 5
TR_ERR_UNSUPPORTED = 6

TR_ALG = {"tvm": 0, "tvme": 1, "tvmw": 2}
TR_PLAN_AUTOTUNE = 1
TR_PLAN_NO_TMA = 2
TR_PLAN_YZ_FUSION = 4
TR_PLAN_THREE_PASS_320 = 8
TR_PLAN_NO_COLUMN_SKIP = 16

EXPORTED = (
    "tr_plan_create", "tr_plan_destroy", "tr_plan_info", "tr_last_error_string", "tr_plan_set_maps",
    "tr_plan_sort_kspace", "tr_plan_unsort_kspace", "tr_nufft_forward", "tr_nufft_adjoint",
    "tr_nufft_forward_bin", "tr_nufft_adjoint_bin", "tr_plan_bin_offset", "tr_pdhg_run",
    "tr_power_iteration", "tr_profile_nufft", "tr_tolerance_sums_noalloc", "tr_conv3d_fwd",
    "tr_conv3d_wgrad_workspace", "tr_conv3d_wgrad", "tr_pdhg_phase", "tr_plan_set_wait_limit",
    "tr_wavelet_forward", "tr_wavelet_adjoint",
)

DEFAULT_WAIT_POLLS = 1 << 20   # bounded mbarrier waits: polls before a wait gives up


class TrError(RuntimeError):
    """A toporecon_b200 call failed; ``code`` is the tr_status value."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[tr_status {code}] {message}")
        self.code = code


class TrNonFinite(TrError, OverflowError):
    """Non-finite tolerance (the reference maps it to an OverflowError retry)."""


class PlanDesc(ctypes.Structure):
    _fields_ = [
        ("img_shape", ctypes.c_int32 * 3),
        ("n_bins", ctypes.c_int32),
        ("bin_counts", ctypes.POINTER(ctypes.c_int64)),
        ("coords", ctypes.POINTER(ctypes.c_float)),
        ("dcf", ctypes.POINTER(ctypes.c_float)),
        ("n_coils", ctypes.c_int32),
        ("n_echoes", ctypes.c_int32),
        ("oversamp", ctypes.c_float),
        ("width", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]


class PlanInfo(ctypes.Structure):
    _fields_ = [
        ("os_shape", ctypes.c_int32 * 3),
        ("total_samples", ctypes.c_int64),
        ("workspace_bytes", ctypes.c_int64),
        ("wavelet_levels", ctypes.c_int32),
        ("wavelet_coeffs", ctypes.c_int64),
        ("fft_line_width", ctypes.c_int32),
        ("spread_columns", ctypes.c_int32),
    ]


class PdhgParams(ctypes.Structure):
    _fields_ = [
        ("algorithm", ctypes.c_int32),
        ("l2_coupling", ctypes.c_int32),
        ("sigma", ctypes.c_float),
        ("tau", ctypes.c_float),
        ("lam_m", ctypes.c_float),
        ("lam_e", ctypes.c_float),
        ("lam_w1", ctypes.c_float),
        ("lam_w2", ctypes.c_float),
        ("use_graph", ctypes.c_int32),
        ("sigma_data", ctypes.c_float),
    ]


class PdhgState(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in
                ("u", "u_bar", "p_m", "p_ex", "p_ey", "p_ez", "p_w1", "p_w2", "w2adj", "q", "y", "g")]


class PdhgShard(ctypes.Structure):
    _fields_ = [
        ("n_bins_global", ctypes.c_int32),
        ("bin_offset", ctypes.c_int32),
        ("u_bar_next", ctypes.c_void_p),
        ("p_m_prev", ctypes.c_void_p),
    ]


_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """Load the library (once); raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is not built; run `python {LIB_PATH.parent.name}/build.py` "
                "(the b200 backend has no CPU fallback)")
        lib = ctypes.CDLL(str(LIB_PATH))
        vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        sig = {
            "tr_plan_create": ([ctypes.POINTER(PlanDesc), ctypes.POINTER(vp)], i32),
            "tr_plan_destroy": ([vp], i32),
            "tr_plan_info": ([vp, ctypes.POINTER(PlanInfo)], i32),
            "tr_last_error_string": ([], ctypes.c_char_p),
            "tr_plan_set_maps": ([vp, vp, vp], i32),
            "tr_plan_sort_kspace": ([vp, i32, vp, vp, i32, vp], i32),
            "tr_plan_unsort_kspace": ([vp, i32, vp, vp, i32, vp], i32),
            "tr_nufft_forward": ([vp, i32, vp, vp, vp], i32),
            "tr_nufft_adjoint": ([vp, i32, vp, vp, vp], i32),
            "tr_nufft_forward_bin": ([vp, i32, vp, vp, vp], i32),
            "tr_nufft_adjoint_bin": ([vp, i32, vp, i32, vp, vp], i32),
            "tr_plan_bin_offset": ([vp, i32, ctypes.POINTER(i64), ctypes.POINTER(i64)], i32),
            "tr_pdhg_run": ([vp, ctypes.POINTER(PdhgState), ctypes.POINTER(PdhgParams), i32, ctypes.c_double,
                             ctypes.POINTER(ctypes.c_double), ctypes.POINTER(i32), vp], i32),
            "tr_power_iteration": ([vp, i32, vp, ctypes.POINTER(ctypes.c_double), vp], i32),
            "tr_profile_nufft": ([vp, i32, i32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                  vp], i32),
            "tr_tolerance_sums_noalloc": ([vp, vp, i64, i32, vp, vp], i32),
            "tr_conv3d_fwd": ([vp, vp, vp, vp, i32, i32, i32, i32, i32, i32, vp], i32),
            "tr_conv3d_wgrad_workspace": ([i32, i32, i32, i32, i32, i32, ctypes.POINTER(ctypes.c_size_t)], i32),
            "tr_conv3d_wgrad": ([vp, vp, vp, i32, i32, i32, i32, i32, i32, vp, ctypes.c_size_t, vp], i32),
            "tr_pdhg_phase": ([vp, ctypes.POINTER(PdhgState), ctypes.POINTER(PdhgParams), ctypes.POINTER(PdhgShard),
                               i32, vp, vp], i32),
            "tr_plan_set_wait_limit": ([vp, i32], i32),
            "tr_wavelet_forward": ([vp, vp, vp, vp], i32),
            "tr_wavelet_adjoint": ([vp, vp, vp, vp], i32),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def last_error() -> str:
    msg = load().tr_last_error_string()
    return msg.decode("utf-8", "replace") if msg else ""


def check(status: int, what: str = "") -> None:
    if status == TR_OK:
        return
    msg = last_error()
    if status == TR_ERR_NONFINITE:
        raise TrNonFinite(status, msg)
    if status == TR_ERR_INVALID_ARG:
        if "bin_index" in msg:
            raise IndexError(msg)
        raise ValueError(msg)
    raise TrError(status, f"{what}: {msg}" if what else msg)
