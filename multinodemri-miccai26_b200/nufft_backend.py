"""NUFFT backends behind the reference's plugin interface, plus the b200 backend.

Mirrors the plugin layer of ``src/toporecon/nufft_backend.py`` in the reference:

* ``NufftBackend``          -- the abstract contract (``:11-52``): ``xp``,
  ``num_bins``, ``to_device``, ``forward(image, bin)``, ``adjoint(ksp, bin)``
  and ``_validate_bin``, whose ``IndexError`` text is part of that contract;
* ``B200NufftBackend``      -- the sm_100a implementation.  ``forward`` /
  ``adjoint`` accept NumPy, CuPy or torch arrays and return the same kind
  (zero-copy through DLPack for device arrays), so the reference's per-call
  sites (``tvme.py:263``, ``:389``) can use it unchanged.  The batched methods
  (``forward_bin`` / ``adjoint_bin``) are the hot path of the b200
  reconstructors;
* ``create_nufft_backend``  -- the registry (``:119-135``) with ``"b200"``
  added.  ``"sigpy"`` hands over to the reference package's own SigPy backend
  when ``toporecon`` and SigPy are importable, and raises ``RuntimeError``
  otherwise; this package carries no SigPy code.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod
from typing import Any, Iterable, Sequence

import numpy as np

from . import _lib


class NufftBackend(ABC):
    """What a reconstructor needs from a NUFFT: per-bin forward and adjoint.

    A backend holds the trajectory of every local motion bin, with coordinates
    already ordered ``[z, y, x]`` in grid units.
    """

    def __init__(self, img_shape: Sequence[int]) -> None:
        self.img_shape = tuple(int(value) for value in img_shape)
        if len(self.img_shape) != 3 or any(value < 1 for value in self.img_shape):
            raise ValueError(f"img_shape must be three positive values: {img_shape}.")

    @property
    @abstractmethod
    def xp(self) -> Any:
        """The array module of the backend's results."""

    @property
    @abstractmethod
    def num_bins(self) -> int:
        """How many motion bins the backend holds trajectories for."""

    @abstractmethod
    def to_device(self, array: Any) -> Any:
        """Return ``array`` on the backend's device, in its array type."""

    @abstractmethod
    def forward(self, image: Any, bin_index: int) -> Any:
        """Non-uniform k-space of one image at the trajectory of one bin."""

    @abstractmethod
    def adjoint(self, kspace: Any, bin_index: int) -> Any:
        """Image-space adjoint of one bin's k-space samples."""

    def _validate_bin(self, bin_index: int) -> int:
        resolved = int(bin_index)
        if not 0 <= resolved < self.num_bins:
            raise IndexError(f"bin_index {resolved} is outside [0, {self.num_bins}).")
        return resolved


# ---------------------------------------------------------------------- helpers
def _device_index(device) -> int:
    if device is None:
        return 0
    if isinstance(device, str):
        import torch
        d = torch.device(device)
        if d.type != "cuda":
            raise ValueError("the b200 backend runs on a CUDA device; got " + device)
        return 0 if d.index is None else int(d.index)
    if hasattr(device, "id"):           # sigpy.Device
        device = device.id
    if type(device).__module__.startswith("torch"):
        if device.type != "cuda":
            raise ValueError("the b200 backend runs on a CUDA device")
        return 0 if device.index is None else int(device.index)
    dev = int(device)
    if dev < 0:
        raise ValueError("the b200 backend runs on a CUDA device; got the CPU device")
    return dev


def _to_host_f32(a) -> np.ndarray:
    if hasattr(a, "detach"):
        return a.detach().to("cpu").numpy().astype(np.float32, copy=False)
    if hasattr(a, "get") and not isinstance(a, np.ndarray):  # CuPy
        a = a.get()
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _kind(a) -> str:
    mod = type(a).__module__.split(".")[0]
    if mod == "torch":
        return "torch"
    if mod == "cupy":
        return "cupy"
    return "numpy"


class B200NufftBackend(NufftBackend):
    """Kaiser-Bessel NUFFT (SigPy 0.1.27 definition) on one B200.

    Parameters mirror the reference's ``SigPyNufftBackend(img_shape,
    coordinates, device)`` (``nufft_backend.py:58-88``);
    ``dcf`` (per-bin density weights), ``n_coils`` and ``n_echoes`` configure
    the batched path used by the b200 reconstructors.  ``tma``, ``fuse_yz`` and
    ``three_pass_320`` select kernel variants for comparison runs (TR_PLAN_NO_TMA,
    TR_PLAN_YZ_FUSION, TR_PLAN_THREE_PASS_320); results agree to float rounding.
    ``column_skip=False`` (TR_PLAN_NO_COLUMN_SKIP) makes the z passes transform
    the grid lines of (y, x) tile columns no sample reaches as well (same bits).
    """

    def __init__(self, img_shape, coordinates, device=0, *, dcf: Iterable | None = None, n_coils: int = 1,
                 n_echoes: int = 1, autotune: bool = False, tma: bool = True, fuse_yz: bool = False,
                 three_pass_320: bool = False, column_skip: bool = True) -> None:
        super().__init__(img_shape)
        import torch
        self._torch = torch
        self.device_index = _device_index(device)
        self.device = torch.device("cuda", self.device_index)
        coords = []
        for index, coordinate in enumerate(coordinates):
            array = coordinate if hasattr(coordinate, "shape") else np.asarray(coordinate)
            if array.ndim < 2 or array.shape[-1] != len(self.img_shape):
                raise ValueError(f"coordinates[{index}] must end in dimension {len(self.img_shape)}, "
                                 f"got {tuple(array.shape)}.")
            coords.append(_to_host_f32(array))
        if not coords:
            raise ValueError("At least one trajectory bin is required.")
        self.bin_shapes = tuple(c.shape[:-1] for c in coords)
        counts = np.array([int(np.prod(s)) for s in self.bin_shapes], dtype=np.int64)
        flat = np.ascontiguousarray(np.concatenate([c.reshape(-1, 3) for c in coords]), dtype=np.float32)
        dcf_flat = None
        if dcf is not None:
            dl = [_to_host_f32(d).reshape(-1) for d in dcf]
            if len(dl) != len(coords) or any(d.size != n for d, n in zip(dl, counts)):
                raise ValueError("dcf must hold one weight per sample of every bin")
            dcf_flat = np.ascontiguousarray(np.concatenate(dl), dtype=np.float32)
        self.n_coils = int(n_coils)
        self.n_echoes = int(n_echoes)
        self._counts = counts
        self._offsets = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64)
        lib = _lib.load()
        desc = _lib.PlanDesc()
        for i in range(3):
            desc.img_shape[i] = self.img_shape[i]
        desc.n_bins = len(coords)
        desc.bin_counts = counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        desc.coords = flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        desc.dcf = dcf_flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if dcf_flat is not None else None
        desc.n_coils = self.n_coils
        desc.n_echoes = self.n_echoes
        desc.oversamp = 1.25
        desc.width = 4
        desc.device = self.device_index
        desc.flags = ((_lib.TR_PLAN_AUTOTUNE if autotune else 0) | (0 if tma else _lib.TR_PLAN_NO_TMA)
                      | (_lib.TR_PLAN_YZ_FUSION if fuse_yz else 0) | (_lib.TR_PLAN_THREE_PASS_320 if three_pass_320 else 0)
                      | (0 if column_skip else _lib.TR_PLAN_NO_COLUMN_SKIP))
        handle = ctypes.c_void_p()
        _lib.check(lib.tr_plan_create(ctypes.byref(desc), ctypes.byref(handle)), "tr_plan_create")
        self._plan = handle
        self._lib = lib
        info = _lib.PlanInfo()
        _lib.check(lib.tr_plan_info(self._plan, ctypes.byref(info)))
        self.os_shape = tuple(info.os_shape)
        self.autotune = bool(autotune)
        self.total_samples = int(info.total_samples)
        self.wavelet_levels = int(info.wavelet_levels)
        self.wavelet_coeffs = int(info.wavelet_coeffs)
        self.has_maps = False

    # ------------------------------------------------------------------ contract
    @property
    def xp(self):
        return self._torch

    @property
    def num_bins(self) -> int:
        return len(self.bin_shapes)

    @property
    def plan(self) -> ctypes.c_void_p:
        return self._plan

    def bin_count(self, b: int) -> int:
        return int(self._counts[b])

    def bin_offset(self, b: int) -> int:
        return int(self._offsets[b])

    def _stream(self):
        return ctypes.c_void_p(self._torch.cuda.current_stream(self.device).cuda_stream)

    def to_device(self, array: Any):
        torch = self._torch
        if isinstance(array, torch.Tensor):
            t = array
        elif _kind(array) == "cupy":
            t = torch.from_dlpack(array)
        else:
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(array)))
        return t.to(device=self.device, dtype=torch.complex64).contiguous()

    def _return_like(self, out, like):
        kind = _kind(like)
        if kind == "torch":
            return out
        if kind == "cupy":
            import cupy
            return cupy.from_dlpack(out)
        return out.cpu().numpy()

    def forward(self, image: Any, bin_index: int) -> Any:
        b = self._validate_bin(bin_index)
        x = self.to_device(image)
        if tuple(x.shape) != self.img_shape:
            raise ValueError(f"image must have shape {self.img_shape}, got {tuple(x.shape)}")
        out = self._torch.empty(self.bin_shapes[b], dtype=self._torch.complex64, device=self.device)
        _lib.check(self._lib.tr_nufft_forward(self._plan, b, ctypes.c_void_p(x.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()), self._stream()), "forward")
        return self._return_like(out, image)

    def adjoint(self, kspace: Any, bin_index: int) -> Any:
        b = self._validate_bin(bin_index)
        y = self.to_device(kspace)
        if int(y.numel()) != self.bin_count(b):
            raise ValueError(f"kspace must hold {self.bin_count(b)} samples for bin {b}, got {int(y.numel())}")
        out = self._torch.empty(self.img_shape, dtype=self._torch.complex64, device=self.device)
        _lib.check(self._lib.tr_nufft_adjoint(self._plan, b, ctypes.c_void_p(y.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr()), self._stream()), "adjoint")
        return self._return_like(out, kspace)

    # ------------------------------------------------------------------ batched path
    def set_maps(self, mps) -> None:
        m = self.to_device(mps)
        if tuple(m.shape) != (self.n_coils,) + self.img_shape:
            raise ValueError(f"maps must be {(self.n_coils,) + self.img_shape}, got {tuple(m.shape)}")
        _lib.check(self._lib.tr_plan_set_maps(self._plan, ctypes.c_void_p(m.data_ptr()), self._stream()))
        self._maps_ref = m
        self.has_maps = True

    def sort_kspace(self, ext, bin_index: int, out=None):
        """(ncol, M_b) acquisition order -> (M_b, ncol) tile-sorted."""
        b = self._validate_bin(bin_index)
        e = self.to_device(ext).reshape(-1, self.bin_count(b))
        ncol = e.shape[0]
        if out is None:
            out = self._torch.empty((self.bin_count(b), ncol), dtype=self._torch.complex64, device=self.device)
        _lib.check(self._lib.tr_plan_sort_kspace(self._plan, b, ctypes.c_void_p(e.data_ptr()),
                                                 ctypes.c_void_p(out.data_ptr()), ncol, self._stream()))
        return out

    def unsort_kspace(self, internal, bin_index: int):
        """(M_b, ncol) tile-sorted -> (ncol, M_b) acquisition order."""
        b = self._validate_bin(bin_index)
        i = internal.reshape(self.bin_count(b), -1)
        ncol = i.shape[1]
        out = self._torch.empty((ncol, self.bin_count(b)), dtype=self._torch.complex64, device=self.device)
        _lib.check(self._lib.tr_plan_unsort_kspace(self._plan, b, ctypes.c_void_p(i.data_ptr()),
                                                   ctypes.c_void_p(out.data_ptr()), ncol, self._stream()))
        return out

    def forward_bin(self, images, bin_index: int, out=None):
        """images (E, Z, Y, X) -> (M_b, E*C) sorted k-space of images[e] * S_c."""
        b = self._validate_bin(bin_index)
        if not self.has_maps:
            raise RuntimeError("set_maps() first")
        x = images.contiguous()
        if out is None:
            out = self._torch.empty((self.bin_count(b), self.n_echoes * self.n_coils), dtype=self._torch.complex64,
                                    device=self.device)
        _lib.check(self._lib.tr_nufft_forward_bin(self._plan, b, ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def adjoint_bin(self, ksp_internal, bin_index: int, use_dcf: bool = True, out=None):
        """(M_b, E*C) sorted k-space -> (E, Z, Y, X) coil-combined images."""
        b = self._validate_bin(bin_index)
        if not self.has_maps:
            raise RuntimeError("set_maps() first")
        k = ksp_internal.contiguous()
        if out is None:
            out = self._torch.empty((self.n_echoes,) + self.img_shape, dtype=self._torch.complex64,
                                    device=self.device)
        _lib.check(self._lib.tr_nufft_adjoint_bin(self._plan, b, ctypes.c_void_p(k.data_ptr()), int(use_dcf),
                                                  ctypes.c_void_p(out.data_ptr()), self._stream()))
        return out

    def power_norm(self, n_iter: int = 30, seed: int = 0, work=None) -> float:
        """sqrt(||A^H W A||) of the batched data operator (every bin, echo and
        coil; W = the plan's density weights) by ``n_iter`` power-iteration
        steps from a seeded random start; FP64 norms (``tr_power_iteration``).
        ``work``: optional (B, Z, Y, X) complex64 start / scratch (one image
        per bin: every echo of a bin sees the same operator)."""
        if not self.has_maps:
            raise RuntimeError("set_maps() first")
        torch = self._torch
        shape = (self.num_bins,) + self.img_shape
        if work is not None and (not work.is_contiguous() or work.numel() != int(np.prod(shape))):
            raise ValueError(f"work must be a contiguous {shape} complex64 tensor")
        if work is None:
            gen = torch.Generator(device=self.device)
            gen.manual_seed(int(seed))
            work = torch.randn(shape, dtype=torch.complex64, device=self.device, generator=gen)
        out = ctypes.c_double(0.0)
        _lib.check(self._lib.tr_power_iteration(self._plan, int(n_iter), ctypes.c_void_p(work.data_ptr()),
                                                ctypes.byref(out), self._stream()), "tr_power_iteration")
        return float(out.value)

    def wavelet_forward(self, images, out=None):
        """W2 analysis (db6, zero mode, PyWavelets' maximum level) of the
        (B, E, Z, Y, X) images -> (B*E, wavelet_coeffs) coefficient trees."""
        torch = self._torch
        x = images.contiguous()
        n_img = self.num_bins * self.n_echoes
        if x.numel() != n_img * int(np.prod(self.img_shape)):
            raise ValueError(f"images must hold {n_img} images of {self.img_shape}")
        if out is None:
            out = torch.empty((n_img, self.wavelet_coeffs), dtype=torch.complex64, device=self.device)
        _lib.check(self._lib.tr_wavelet_forward(self._plan, ctypes.c_void_p(x.data_ptr()),
                                                ctypes.c_void_p(out.data_ptr()), self._stream()), "wavelet_forward")
        return out

    def wavelet_adjoint(self, coeffs, out=None):
        """waverec3 of (B*E, wavelet_coeffs) trees cropped to (B, E, Z, Y, X)."""
        torch = self._torch
        c = coeffs.contiguous()
        if out is None:
            out = torch.empty((self.num_bins, self.n_echoes) + self.img_shape, dtype=torch.complex64,
                              device=self.device)
        _lib.check(self._lib.tr_wavelet_adjoint(self._plan, ctypes.c_void_p(c.data_ptr()),
                                                ctypes.c_void_p(out.data_ptr()), self._stream()), "wavelet_adjoint")
        return out

    def set_wait_limit(self, polls: int = _lib.DEFAULT_WAIT_POLLS) -> None:
        """Polls before a bounded device wait gives up (0: every wait gives up at
        once, the next PDHG call then raises with TR_ERR_TIMEOUT)."""
        _lib.check(self._lib.tr_plan_set_wait_limit(self._plan, int(polls)), "tr_plan_set_wait_limit")

    STAGES = ("fwd_x", "fwd_y", "fwd_z", "interp", "spread", "adj_z", "adj_y", "adj_x", "fwd_yz", "adj_zy")
    # the stages one batched forward + adjoint runs, with and without the fused y / z passes
    PIPELINE_FUSED = ("fwd_x", "fwd_yz", "interp", "spread", "adj_zy", "adj_x")
    PIPELINE_SEPARATE = ("fwd_x", "fwd_y", "fwd_z", "interp", "spread", "adj_z", "adj_y", "adj_x")

    def profile(self, bin_index: int = 0, reps: int = 5) -> dict:
        """CUDA-event time (ms) and algorithmic bytes of each NUFFT stage of one
        bin; ``fwd_yz`` / ``adj_zy`` (the fused y + z passes) are absent when the
        plan runs the separate passes.  ``pipeline(profile)`` lists the stages
        the solver actually runs."""
        b = self._validate_bin(bin_index)
        ms = (ctypes.c_double * 10)()
        by = (ctypes.c_double * 10)()
        _lib.check(self._lib.tr_profile_nufft(self._plan, b, int(reps), ms, by, self._stream()), "profile")
        self._torch.cuda.synchronize(self.device)
        return {name: {"ms": ms[i], "bytes": by[i], "gbs": by[i] / (ms[i] * 1e6) if ms[i] > 0 else 0.0}
                for i, name in enumerate(self.STAGES) if i < 8 or ms[i] > 0}

    @classmethod
    def pipeline(cls, prof: dict) -> tuple:
        return cls.PIPELINE_FUSED if "fwd_yz" in prof and "adj_zy" in prof else cls.PIPELINE_SEPARATE

    @property
    def spread_columns(self) -> int:
        """k-space columns per gridding CTA (the autotuner's choice once it has run)."""
        info = _lib.PlanInfo()
        _lib.check(self._lib.tr_plan_info(self._plan, ctypes.byref(info)))
        return int(info.spread_columns)

    def close(self) -> None:
        if getattr(self, "_plan", None):
            self._lib.tr_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def create_nufft_backend(name: str, *, img_shape: Sequence[int], coordinates: Iterable, device: Any,
                         **kwargs) -> NufftBackend:
    """Construct a registered backend without conditionals in algorithms."""
    normalized = name.strip().lower()
    if normalized == "sigpy":
        try:
            from toporecon.nufft_backend import SigPyNufftBackend
        except ImportError as exc:
            raise RuntimeError("the 'sigpy' backend is the reference toporecon package's own SigPy "
                               f"implementation, which cannot be imported here ({exc}); use 'b200'") from exc
        return SigPyNufftBackend(img_shape=img_shape, coordinates=coordinates, device=device)
    if normalized == "b200":
        return B200NufftBackend(img_shape, coordinates, device, **kwargs)
    raise ValueError(f"Unknown NUFFT backend {name!r}. Available backends: sigpy, b200.")
