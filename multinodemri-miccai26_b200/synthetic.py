"""Seeded synthetic motion-resolved multi-echo cones datasets.

The reference is run on a 3-D multi-echo cones liver dataset that is not
available here, so every workload is a seeded synthetic stand-in with the
reference's data contract (k-space ``(E, C, TR, RO)``, trajectory
``(TR, RO, 3)`` in grid units ordered z, y, x, density ``(TR, RO)``,
respiratory signal ``(TR,)``; ``data/dataset.py:54-88``):

* 3-D cones: ``TR`` interleaves of ``RO`` points, cone axes spread uniformly
  in ``cos(theta)`` and golden-angle azimuth, acquired in a shuffled order,
  ``|k| < n/2`` per axis;
* phantom: random ellipsoids whose z position follows the respiratory
  displacement (0 to ``shift_mm`` mm, 1 mm voxels), per-ellipsoid
  ``R2*`` and off-resonance giving ``exp(-TE R2*) exp(2 pi i df TE)``;
* coil maps: Gaussian magnitude centred on a cylinder, random linear phase,
  unit root-sum-of-squares;
* respiratory signal: a 4 s sinusoid plus noise, amplitude-binned with the
  reference's percentile rule (``algorithms/tvme.py:853-881``), or Dirichlet
  bin sizes for the uneven-bin workload;
* density: ``|k|^2`` (normalised radius), clipped, divided by its maximum;
* noise: complex Gaussian, sigma = ``noise_frac`` x max |k-space|.

The k-space simulation itself is delegated to a caller-provided forward
operator so that large workloads are simulated by the b200 NUFFT on the GPU.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field, replace
from typing import Callable, Optional

import numpy as np


@dataclass(frozen=True)
class SyntheticConfig:
    name: str
    img_shape: tuple            # (Z, Y, X)
    n_coils: int
    n_echoes: int
    n_bins: int
    n_interleaves: int
    n_readout: int
    algorithm: str = "tvme"
    l2_coupling: bool = False
    lam: float = 1e-5
    max_iter: int = 300
    tol: float = 1e-3
    te0: float = 1.2e-3
    dte: float = 1.1e-3
    r2_range: tuple = (20.0, 80.0)
    df_range: tuple = (-50.0, 50.0)
    n_ellipsoids: int = 6
    shift_mm: float = 8.0
    noise_frac: float = 0.01
    resp_period_s: float = 4.0
    scan_time_s: float = 24.0
    binning: str = "amplitude"   # or "dirichlet"
    dirichlet_alpha: float = 2.0
    seed: int = 0


CONFIGS = {
    # TVM plain PDHG, CPU-runnable.
    "tvm-64": SyntheticConfig("tvm-64", (48, 64, 64), 4, 1, 6, 512, 400, algorithm="tvm",
                              max_iter=100, tol=0.0),
    # TVME with L2 coupling.
    "tvme-128": SyntheticConfig("tvme-128", (96, 128, 128), 8, 4, 6, 1024, 600, algorithm="tvme",
                                l2_coupling=True),
    # TVMW with db1 echo and 3-level db6 spatial wavelets.
    "tvmw-160": SyntheticConfig("tvmw-160", (112, 160, 160), 12, 6, 6, 1600, 700, algorithm="tvmw"),
    # Batched uneven TVME, Dirichlet(2) bin sizes.
    "tvme-256-dirichlet": SyntheticConfig("tvme-256-dirichlet", (128, 256, 256), 16, 6, 8, 4096, 800,
                                          algorithm="tvme", binning="dirichlet"),
    # Warm-start evaluation workload, timed to tol 1e-3: the cap sits well above
    # the iteration where the power step rule meets the tolerance (about 410).
    "tvme-256": SyntheticConfig("tvme-256", (128, 256, 256), 16, 6, 6, 4096, 800, algorithm="tvme",
                                max_iter=1000),
    # Warm-start training phantoms.
    "warm-96": SyntheticConfig("warm-96", (64, 96, 96), 8, 4, 6, 768, 480, algorithm="tvme"),
}


def scaled(cfg: SyntheticConfig, factor: float, **kw) -> SyntheticConfig:
    """Shrink a workload isotropically (used for quick tests)."""
    shape = tuple(max(8, int(round(n * factor / 4)) * 4) for n in cfg.img_shape)
    n_int = max(16, int(cfg.n_interleaves * factor * factor))
    n_ro = max(16, int(cfg.n_readout * factor))
    return replace(cfg, name=cfg.name + f"-x{factor:g}", img_shape=shape, n_interleaves=n_int,
                   n_readout=n_ro, **kw)


# ------------------------------------------------------------------ trajectory
def cones_trajectory(img_shape, n_interleaves: int, n_readout: int, rng: np.random.Generator) -> np.ndarray:
    """(TR, RO, 3) float32 zyx grid units, |k_axis| < n_axis/2."""
    Z, Y, X = img_shape
    i = np.arange(n_interleaves, dtype=np.float64)
    cos_t = 1.0 - 2.0 * (i + 0.5) / n_interleaves
    theta = np.arccos(cos_t)
    phi0 = (i * math.pi * (3.0 - math.sqrt(5.0))) % (2 * math.pi)
    t = np.linspace(0.0, 1.0, n_readout, dtype=np.float64)
    r = t  # constant radial speed
    turns = 2.0 + 6.0 * np.sin(theta)  # more twist on wide cones
    phi = phi0[:, None] + 2 * math.pi * turns[:, None] * r[None, :]
    st = np.sin(theta)[:, None]
    dz = np.cos(theta)[:, None] * np.ones_like(r)[None, :]
    dy = st * np.sin(phi)
    dx = st * np.cos(phi)
    kmax = 0.5 - 1e-4
    k = np.stack([dz * r * Z * kmax, dy * r * Y * kmax, dx * r * X * kmax], axis=-1)
    order = rng.permutation(n_interleaves)
    return k[order].astype(np.float32)


def density(coord: np.ndarray, img_shape) -> np.ndarray:
    kn = coord.astype(np.float64) / (np.asarray(img_shape, dtype=np.float64) / 2.0)
    r2 = np.sum(kn * kn, axis=-1)
    d = np.clip(r2, 1e-4, 1.0)
    return (d / d.max()).astype(np.float32)


# ------------------------------------------------------------------ phantom
@dataclass
class Ellipsoid:
    center: np.ndarray  # zyx voxels relative to the grid centre
    axes: np.ndarray    # semi-axes zyx voxels
    rho: float
    r2: float
    df: float


def random_ellipsoids(cfg: SyntheticConfig, rng: np.random.Generator) -> list:
    shp = np.asarray(cfg.img_shape, dtype=np.float64)
    out = []
    for _ in range(cfg.n_ellipsoids):
        axes = shp * rng.uniform(0.08, 0.25, size=3)
        center = shp * rng.uniform(-0.22, 0.22, size=3)
        out.append(Ellipsoid(center=center, axes=axes, rho=float(rng.uniform(0.4, 1.0)),
                             r2=float(rng.uniform(*cfg.r2_range)), df=float(rng.uniform(*cfg.df_range))))
    return out


def render_phantom(cfg: SyntheticConfig, ells: list, shifts_mm: np.ndarray) -> np.ndarray:
    """(B, E, Z, Y, X) complex64 images; bin b's ellipsoids move by shifts_mm[b] in z."""
    Z, Y, X = cfg.img_shape
    B, E = len(shifts_mm), cfg.n_echoes
    zz = (np.arange(Z) - Z // 2).astype(np.float32)[:, None, None]
    yy = (np.arange(Y) - Y // 2).astype(np.float32)[None, :, None]
    xx = (np.arange(X) - X // 2).astype(np.float32)[None, None, :]
    te = cfg.te0 + cfg.dte * np.arange(E)
    out = np.zeros((B, E, Z, Y, X), dtype=np.complex64)
    for b in range(B):
        for el in ells:
            cz, cy, cx = el.center
            az, ay, ax = el.axes
            m = (((zz - (cz + shifts_mm[b])) / az) ** 2 + ((yy - cy) / ay) ** 2 + ((xx - cx) / ax) ** 2) <= 1.0
            for e in range(E):
                val = el.rho * math.exp(-te[e] * el.r2) * complex(math.cos(2 * math.pi * el.df * te[e]),
                                                                 math.sin(2 * math.pi * el.df * te[e]))
                out[b, e][m] += np.complex64(val)
    return out


def coil_maps(img_shape, n_coils: int, rng: np.random.Generator) -> np.ndarray:
    """(C, Z, Y, X) complex64, Gaussian magnitude on a cylinder, unit SOS."""
    Z, Y, X = img_shape
    zz = ((np.arange(Z) - Z // 2) / (Z / 2)).astype(np.float32)[:, None, None]
    yy = ((np.arange(Y) - Y // 2) / (Y / 2)).astype(np.float32)[None, :, None]
    xx = ((np.arange(X) - X // 2) / (X / 2)).astype(np.float32)[None, None, :]
    rings = 2 if n_coils >= 8 else 1
    per_ring = int(math.ceil(n_coils / rings))
    maps = np.zeros((n_coils,) + tuple(img_shape), dtype=np.complex64)
    for c in range(n_coils):
        ring = c // per_ring
        ang = 2 * math.pi * (c % per_ring) / per_ring + ring * math.pi / per_ring
        cy, cx = 1.1 * math.sin(ang), 1.1 * math.cos(ang)
        cz = 0.0 if rings == 1 else (-0.5 if ring == 0 else 0.5)
        width = 0.8
        mag = np.exp(-(((zz - cz) ** 2) + (yy - cy) ** 2 + (xx - cx) ** 2) / (2 * width * width))
        g = rng.uniform(-1.5, 1.5, size=3)
        phase = g[0] * zz + g[1] * yy + g[2] * xx + rng.uniform(0, 2 * math.pi)
        maps[c] = (mag * np.exp(1j * phase)).astype(np.complex64)
    sos = np.sqrt(np.sum(np.abs(maps) ** 2, axis=0))
    sos = np.maximum(sos, np.float32(1e-12))
    return (maps / sos[None]).astype(np.complex64)


# ------------------------------------------------------------------ respiration & bins
def respiratory_signal(n_tr: int, cfg: SyntheticConfig, rng: np.random.Generator) -> np.ndarray:
    t = np.arange(n_tr, dtype=np.float64) * (cfg.scan_time_s / n_tr)
    s = np.sin(2 * math.pi * t / cfg.resp_period_s) + 0.05 * rng.standard_normal(n_tr)
    return s.astype(np.float32)


def percentile_bin_edges(resp: np.ndarray, n_bins: int, margin: float = 0.0) -> np.ndarray:
    """Reference rule: np.percentile(resp, linspace(margin, 100 - margin, B + 1))."""
    return np.percentile(resp, np.linspace(0 + margin, 100 - margin, n_bins + 1))


def assign_bins(resp: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """-1 for TRs outside every half-open bin [edge_b, edge_b+1) (the max is dropped)."""
    out = np.full(resp.shape, -1, dtype=np.int64)
    for b in range(len(edges) - 1):
        out[(resp >= edges[b]) & (resp < edges[b + 1])] = b
    return out


# ------------------------------------------------------------------ dataset
@dataclass
class Dataset:
    cfg: SyntheticConfig
    coord: np.ndarray        # (TR, RO, 3) float32 zyx grid units
    dcf: np.ndarray          # (TR, RO) float32 (max-normalised)
    resp: np.ndarray         # (TR,) float32
    tr_bin: np.ndarray       # (TR,) int64 bin index or -1
    mps: np.ndarray          # (C, Z, Y, X) complex64, unit SOS
    truth: np.ndarray        # (B, E, Z, Y, X) complex64
    ksp: Optional[np.ndarray] = None   # (E, C, TR, RO) complex64, max-normalised
    meta: dict = field(default_factory=dict)

    def bin_indices(self, b: int) -> np.ndarray:
        return np.nonzero(self.tr_bin == b)[0]

    def bin_coords(self):
        return [self.coord[self.bin_indices(b)] for b in range(self.cfg.n_bins)]

    def bin_dcf(self):
        return [self.dcf[self.bin_indices(b)] for b in range(self.cfg.n_bins)]

    def bin_ksp(self):
        return [self.ksp[:, :, self.bin_indices(b)] for b in range(self.cfg.n_bins)]


def make_geometry(cfg: SyntheticConfig) -> Dataset:
    """Everything except k-space: trajectory, density, binning, maps, phantom."""
    rng = np.random.default_rng(cfg.seed)
    coord = cones_trajectory(cfg.img_shape, cfg.n_interleaves, cfg.n_readout, rng)
    dcf = density(coord, cfg.img_shape)
    resp = respiratory_signal(cfg.n_interleaves, cfg, rng)
    if cfg.binning == "dirichlet":
        frac = rng.dirichlet([cfg.dirichlet_alpha] * cfg.n_bins)
        counts = np.maximum(1, np.floor(frac * cfg.n_interleaves).astype(np.int64))
        while counts.sum() > cfg.n_interleaves:
            counts[np.argmax(counts)] -= 1
        counts[np.argmin(counts)] += cfg.n_interleaves - counts.sum()
        tr_bin = np.repeat(np.arange(cfg.n_bins), counts)
        tr_bin = tr_bin[rng.permutation(cfg.n_interleaves)]
        edges = None
    else:
        edges = percentile_bin_edges(resp, cfg.n_bins)
        tr_bin = assign_bins(resp, edges)
    # displacement of each bin: mean normalised respiratory amplitude of its TRs
    lo, hi = float(resp.min()), float(resp.max())
    disp = (resp - lo) / max(hi - lo, 1e-12) * cfg.shift_mm
    shifts = np.array([float(disp[tr_bin == b].mean()) if np.any(tr_bin == b) else 0.0
                       for b in range(cfg.n_bins)])
    if cfg.binning == "dirichlet":
        shifts = cfg.shift_mm * 0.5 * (1 - np.cos(math.pi * np.arange(cfg.n_bins) / max(1, cfg.n_bins - 1)))
    ells = random_ellipsoids(cfg, rng)
    truth = render_phantom(cfg, ells, shifts)
    mps = coil_maps(cfg.img_shape, cfg.n_coils, rng)
    return Dataset(cfg=cfg, coord=coord, dcf=dcf, resp=resp, tr_bin=tr_bin, mps=mps, truth=truth,
                   meta={"bin_edges": None if edges is None else edges.tolist(),
                         "shifts_mm": shifts.tolist(), "noise_seed": cfg.seed + 1})


def simulate_kspace_b200(ds: Dataset, device=0) -> Dataset:
    """``simulate_kspace`` with the b200 batched forward NUFFT on the GPU."""
    import torch

    from .nufft_backend import B200NufftBackend
    cfg = ds.cfg
    E, C = cfg.n_echoes, cfg.n_coils
    TR, RO = ds.coord.shape[:2]
    coords = [ds.coord[ds.bin_indices(b)].reshape(-1, 3) for b in range(cfg.n_bins)]
    be = B200NufftBackend(cfg.img_shape, [c if c.size else np.zeros((1, 3), np.float32) for c in coords], device,
                          n_coils=C, n_echoes=E)
    be.set_maps(ds.mps)
    ksp = np.zeros((E, C, TR, RO), dtype=np.complex64)
    for b in range(cfg.n_bins):
        idx = ds.bin_indices(b)
        if idx.size == 0:
            continue
        truth = torch.from_numpy(ds.truth[b]).to(be.device)
        y = be.unsort_kspace(be.forward_bin(truth, b), b)          # (E*C, M_b)
        ksp[:, :, idx] = y.reshape(E, C, idx.size, RO).cpu().numpy()
    be.close()
    rng = np.random.default_rng(ds.meta["noise_seed"])
    sigma = cfg.noise_frac * float(np.abs(ksp).max())
    for e in range(E):   # per echo to bound host memory
        noise = rng.standard_normal((C, TR, RO, 2), dtype=np.float32)
        ksp[e] += (sigma / math.sqrt(2.0)) * (noise[..., 0] + 1j * noise[..., 1]).astype(np.complex64)
    m = float(np.abs(ksp).max())
    if m > 0:
        ksp /= np.float32(m)
    ds.ksp = ksp
    return ds


def simulate_kspace(ds: Dataset, forward: Callable[[np.ndarray, np.ndarray], np.ndarray]) -> Dataset:
    """Fill ``ds.ksp`` with noisy, max-normalised k-space.

    ``forward(images (E*C, Z, Y, X) complex64, coords (M, 3)) -> (E*C, M)``
    simulates one bin; TRs outside every bin get zeros (they are never used).
    """
    cfg = ds.cfg
    E, C = cfg.n_echoes, cfg.n_coils
    TR, RO = ds.coord.shape[:2]
    ksp = np.zeros((E, C, TR, RO), dtype=np.complex64)
    for b in range(cfg.n_bins):
        idx = ds.bin_indices(b)
        if idx.size == 0:
            continue
        imgs = (ds.truth[b][:, None] * ds.mps[None]).reshape((E * C,) + tuple(cfg.img_shape))
        y = forward(imgs.astype(np.complex64), ds.coord[idx].reshape(-1, 3))
        ksp[:, :, idx] = np.asarray(y).reshape(E, C, idx.size, RO)
    rng = np.random.default_rng(ds.meta["noise_seed"])
    sigma = cfg.noise_frac * float(np.abs(ksp).max())
    noise = rng.standard_normal(ksp.shape, dtype=np.float32) + 1j * rng.standard_normal(ksp.shape, dtype=np.float32)
    ksp += (sigma / math.sqrt(2.0)) * noise.astype(np.complex64)
    m = float(np.abs(ksp).max())
    if m > 0:
        ksp /= np.float32(m)
    ds.ksp = ksp
    return ds
