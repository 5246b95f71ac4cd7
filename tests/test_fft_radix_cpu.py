"""Host check of the register DFT butterflies of ``csrc/tr_fft.cuh``.

Every FFT stage of the NUFFT kernels applies ``Dft<R>::run`` to the R values a
thread holds: radices 2-8 for the default plan, and the composite radices of
the two-pass plan (16 = 4 x 4 Cooley-Tukey with W16 twiddles; 10 = 2 x 5 and
20 = 4 x 5 by the Good-Thomas prime-factor maps).  ``tests/native/
dft_radix_host.cu`` runs them on the host (their scalar fallbacks, the same
arithmetic as the packed device forms) in both directions; this test compares
each with numpy's FFT.  Needs nvcc, no GPU.
"""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "dft_radix_host.cu"
RADICES = (2, 3, 4, 5, 7, 8, 10, 16, 20)


@pytest.fixture(scope="module")
def dft_output(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    exe = tmp_path_factory.mktemp("dft") / "dft_radix_host"
    subprocess.run([nvcc, "-std=c++17", "-x", "cu", "-Wno-deprecated-gpu-targets", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "multinodemri-miccai26_b200" / "csrc"), str(SRC), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    res, i = {}, 0
    while i < len(out) and out[i]:
        _, r, inv = out[i].split()
        r, inv = int(r), int(inv)
        vals = [complex(*map(float, ln.split())) for ln in out[i + 1:i + 1 + 2 * r]]
        res[(r, inv)] = (np.array(vals[:r]), np.array(vals[r:]))
        i += 1 + 2 * r
    return res


@pytest.mark.parametrize("inv", (0, 1))
@pytest.mark.parametrize("radix", RADICES)
def test_register_dft_matches_numpy(dft_output, radix, inv):
    x, y = dft_output[(radix, inv)]
    ref = np.fft.ifft(x) * radix if inv else np.fft.fft(x)       # unnormalised both ways
    err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
    assert err < 3e-7, (radix, inv, err)
