"""Write a tiny synthetic dataset in the reference's on-disk format (CFL + txt)."""

import numpy as np

from _fixtures import pkg


def write_dataset(root, shape=(16, 20, 24), C=3, E=2, B=3, TR=60, RO=24, seed=7, voxel=(1.5, 1.2, 1.0)):
    syn = pkg("synthetic")
    cfl = pkg("cfl")
    from oracle import nufft as onf
    cfg = syn.SyntheticConfig("cli", tuple(shape), C, E, B, TR, RO, seed=seed, n_ellipsoids=3)
    ds = syn.make_geometry(cfg)
    syn.simulate_kspace(ds, lambda imgs, k: onf.nufft(imgs, k).astype(np.complex64))
    Z, Y, X = shape
    (root / "imageDim.txt").write_text(f"{X}:{Y}:{Z}\n")
    (root / "voxelSize.txt").write_text(f"{voxel[2]}:{voxel[1]}:{voxel[0]}\n")
    # raw trajectory: physical units, xyz order (the reference scales by voxel * n, reverses xyz -> zyx)
    scale = np.array(voxel) * np.array(shape)            # zyx
    phys = (ds.coord / scale.astype(np.float32))[..., ::-1]
    cfl.write(root / "ktraj", phys.astype(np.complex64))
    cfl.write(root / "dens", (ds.dcf * 3.0).astype(np.complex64))
    cfl.write(root / "resp", ds.resp.astype(np.complex64))
    cfl.write(root / "ksp", (ds.ksp * 5.0).reshape(1, 1, 1, E, 1, C, TR, RO, 1))
    cfl.write(root / "mps", (ds.mps * 2.0).reshape(1, 1, 1, 1, C, Z, Y, X))
    return ds
