"""Respiratory self-navigation signal (the reference's ``toporecon resp``).

Restates ``src/toporecon/preprocessing/respiratory.py:35-114`` of the
reference with the same interface and results:

* the navigator is the magnitude of each trajectory's first readout sample,
  per (echo, coil), with its mean removed;
* every trace is low-passed (Butterworth order 10 at 2 Hz) and then
  high-passed (order 5 at 0.1 Hz), both forward-backward (zero phase), at the
  sampling rate 1 / TR;
* the coils of each echo are combined by their first principal component
  (largest singular value times its right singular vector), then the echoes
  the same way;
* the result is scaled to [0, 1].

It is a host step (a few thousand samples per trace): the reference runs it in
NumPy / SciPy on the CPU, and so does this module.  The motion-bin edges that
the reconstructors derive from it are in ``algorithms/_common.py``.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import cfl as _cfl


@dataclass(frozen=True)
class RespiratoryConfig:
    """Band edges (Hz) and Butterworth orders of the navigator filter."""

    low_cut_hz: float = 0.1
    high_cut_hz: float = 2.0
    low_pass_order: int = 10
    high_pass_order: int = 5

    def validate(self, sampling_rate_hz: float) -> None:
        nyquist = sampling_rate_hz / 2
        if not self.low_cut_hz > 0:
            raise ValueError(f"low_cut_hz has to be above 0 Hz, got {self.low_cut_hz}")
        if not self.high_cut_hz > self.low_cut_hz:
            raise ValueError(f"the pass band is empty: high_cut_hz {self.high_cut_hz} <= low_cut_hz "
                             f"{self.low_cut_hz}")
        if not self.high_cut_hz < nyquist:
            raise ValueError(f"high_cut_hz {self.high_cut_hz} is not below the Nyquist frequency {nyquist} Hz "
                             f"of a {sampling_rate_hz} Hz navigator")


def _leading_component(rows: np.ndarray) -> np.ndarray:
    """sigma_1 v_1 of the SVD of ``rows`` (n, T): the principal time course."""
    _, sv, vt = np.linalg.svd(rows, full_matrices=False)
    return sv[0] * vt[0]


def estimate_respiratory_signal(kspace: np.ndarray, tr_seconds: float, *,
                                config: RespiratoryConfig | None = None) -> np.ndarray:
    """Respiratory signal in [0, 1], one value per trajectory (float32).

    ``kspace``: (echo, coil, trajectory, readout); the first readout sample of
    each trajectory is the navigator.  ``tr_seconds``: the repetition time.
    """
    try:
        from scipy import signal
    except ImportError as exc:  # scipy is a dependency of this package
        raise RuntimeError("respiratory signal estimation needs SciPy") from exc
    data = np.asarray(kspace)
    if data.ndim != 4:
        raise ValueError(f"expected k-space of shape (echo, coil, trajectory, readout), got {data.shape}")
    if not tr_seconds > 0:
        raise ValueError(f"the repetition time has to be positive, got {tr_seconds}")
    cfg = config or RespiratoryConfig()
    fs = 1.0 / float(tr_seconds)
    cfg.validate(fs)
    nav = np.abs(data[..., 0])                                   # (E, C, T), float32 for complex64 input
    nav = nav - nav.mean(axis=-1, keepdims=True, dtype=nav.dtype)
    low = signal.butter(cfg.low_pass_order, cfg.high_cut_hz, "low", fs=fs, output="sos")
    high = signal.butter(cfg.high_pass_order, cfg.low_cut_hz, "high", fs=fs, output="sos")
    band = signal.sosfiltfilt(high, signal.sosfiltfilt(low, nav, axis=-1), axis=-1).astype(np.float32)
    per_echo = np.stack([_leading_component(band[e]) for e in range(band.shape[0])]).astype(np.float32)
    resp = per_echo[0] if per_echo.shape[0] == 1 else _leading_component(per_echo)
    lo, hi = float(resp.min()), float(resp.max())
    if hi - lo <= np.finfo(np.float32).eps:
        raise ValueError("the respiratory signal is flat; it cannot be scaled to [0, 1]")
    return ((resp - lo) / (hi - lo)).astype(np.float32)


def estimate_respiratory_from_dataset(input_directory, output_directory, *,
                                      config: RespiratoryConfig | None = None) -> Path:
    """Read ``ksp`` and ``tr.txt`` of a raw dataset directory and write
    ``resp.hdr/.cfl`` (trajectories x 1) into ``output_directory``."""
    root = Path(input_directory).expanduser().resolve()
    need = [root / "ksp.hdr", root / "ksp.cfl", root / "tr.txt"]
    missing = [str(p) for p in need if not p.is_file()]
    if missing:
        raise FileNotFoundError("the dataset lacks " + ", ".join(missing))
    raw = _cfl.read(root / "ksp", mmap=True)
    E, C, T, R = _cfl.kspace_layout(raw.shape)
    ksp = np.asarray(raw).reshape(E, C, T, R)
    tr = float((root / "tr.txt").read_text(encoding="utf-8").strip())
    resp = estimate_respiratory_signal(ksp, tr, config=config)
    out = Path(output_directory).expanduser() / "resp"
    _cfl.write(out, resp[:, None].astype(np.complex64))
    return out
