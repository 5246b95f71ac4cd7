"""Golden vectors for the host steps either side of the PDHG path, made by the
reference's own code.

    python tests/golden/make_golden_host.py /path/to/reference

* ``resp.npz``: seeded synthetic navigator k-space (3 echoes x 4 coils x 1,200
  trajectories x 1 readout point, a 4 s breathing modulation of the first
  readout sample plus a slow drift and noise) and the output of the
  reference's ``estimate_respiratory_signal`` (``preprocessing/respiratory.py:35-114``)
  at TR = 5 ms and 8 ms;
* ``stitch.npz``: a 2 (motion) x 3 (echo) grid of seeded shards and the image
  the reference's ``stitch`` (``postprocessing/stitch.py:191-256``) assembles
  from them.

The reference's modules for these two steps need only NumPy / SciPy, so they
import here without its GPU dependencies.
"""

from __future__ import annotations

import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def navigator_kspace(seed: int, E=3, C=4, T=1200, R=1, tr=5e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    t = np.arange(T) * tr
    breath = np.sin(2 * np.pi * t / 4.0) + 0.3 * np.sin(2 * np.pi * t / 2.0 + 0.4)
    drift = 0.5 * t / t[-1]
    gains = rng.uniform(0.5, 2.0, size=(E, C))
    ksp = (rng.standard_normal((E, C, T, R)) + 1j * rng.standard_normal((E, C, T, R))).astype(np.complex64) * 0.05
    dc = 10.0 + gains[..., None] * (breath + drift)[None, None] + 0.05 * rng.standard_normal((E, C, T))
    ksp[..., 0] = (dc * np.exp(1j * rng.uniform(0, 2 * np.pi, size=(E, C, 1)))).astype(np.complex64)
    return ksp


def main(reference: str) -> None:
    sys.path.insert(0, str(Path(reference) / "src"))
    from toporecon.postprocessing.stitch import stitch as ref_stitch
    from toporecon.preprocessing.respiratory import estimate_respiratory_signal
    from toporecon.data import cfl as ref_cfl

    out = {}
    for i, tr in enumerate((5e-3, 8e-3)):
        ksp = navigator_kspace(100 + i, tr=tr)
        out[f"ksp{i}"] = ksp
        out[f"tr{i}"] = np.float64(tr)
        out[f"resp{i}"] = estimate_respiratory_signal(ksp, tr)
    np.savez_compressed(HERE / "resp.npz", **out)

    rng = np.random.default_rng(7)
    B, E, Z, Y, X = 4, 5, 3, 4, 6
    full = (rng.standard_normal((B, 1, 1, E, 1, 1, Z, Y, X))
            + 1j * rng.standard_normal((B, 1, 1, E, 1, 1, Z, Y, X))).astype(np.complex64)
    bins, echoes = [(0, 1), (2, 3)], [(0, 1), (2, 3), (4, 4)]
    with tempfile.TemporaryDirectory() as d:
        root = Path(d)
        for b0, b1 in bins:
            for e0, e1 in echoes:
                ref_cfl.write_cfl(root / f"img_e{e0}-{e1}_m{b0}-{b1}", full[b0:b1 + 1, :, :, e0:e1 + 1])
        man = {"output_stem": "img", "parameters": {"num_bins": B, "num_echoes": E},
               "distributed": {"motion_groups": len(bins), "echo_groups": len(echoes)}}
        (root / "run_manifest.json").write_text(json.dumps(man), encoding="utf-8")
        base = ref_stitch(root)
        image = ref_cfl.read_cfl(base)
    np.savez_compressed(HERE / "stitch.npz", image=image, bins=np.array(bins), echoes=np.array(echoes))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden_host.py <path to the reference source tree>")
    main(sys.argv[1])
