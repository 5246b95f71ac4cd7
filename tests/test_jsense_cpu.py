"""JSENSE restatement (oracle) and the b200 entry point's argument checks, on CPU."""

import numpy as np
import pytest

from _fixtures import pkg
from oracle import jsense as oj
from oracle import nufft as onf


def _problem(shape=(24, 24, 24), coils=4, cones=160, readout=120, seed=0):
    syn = pkg("synthetic")
    rng = np.random.default_rng(seed)
    coord = syn.cones_trajectory(shape, cones, readout, rng).reshape(-1, 3)
    dcf = syn.density(coord, shape)
    mps = syn.coil_maps(shape, coils, rng)
    zz, yy, xx = np.meshgrid(*[np.arange(n) - n // 2 for n in shape], indexing="ij")
    img = (((zz / (0.38 * shape[0])) ** 2 + (yy / (0.4 * shape[1])) ** 2 + (xx / (0.35 * shape[2])) ** 2) < 1)
    img = img.astype(np.complex64)
    y = onf.nufft(mps * img[None], coord)
    return coord, dcf, mps, img, y


def rss(a):
    return a / np.sqrt(np.sum(np.abs(a) ** 2, 0, keepdims=True) + 1e-12)


def test_oracle_jsense_recovers_smooth_maps():
    coord, dcf, mps, img, y = _problem()
    maps = oj.jsense(y, coord, dcf, ker_width=6, calib_width=12, max_iter=2, inner=4)
    assert maps.shape == (4, 12, 12, 12)
    full = oj.resize_maps(maps, img.shape)
    corr = np.abs(np.sum(np.conj(rss(full)) * rss(mps), 0))[img != 0]
    assert np.median(corr) > 0.99, np.median(corr)


def test_cg_solves_small_spd_system():
    rng = np.random.default_rng(1)
    a = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    h = a.conj().T @ a + 0.1 * np.eye(6)
    b = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    x = oj.cg(lambda v: h @ v, b, np.zeros(6, complex), 12)
    np.testing.assert_allclose(h @ x, b, rtol=1e-8, atol=1e-8)


def test_entry_point_rejects_mismatched_shapes():
    js = pkg("jsense")
    k = np.zeros((1, 2, 8, 10), np.complex64)
    with pytest.raises(ValueError, match="k-space must have shape"):
        js.estimate_sensitivity_maps(k[0], np.zeros((8, 10, 3)), np.ones((8, 10)), image_shape_zyx=(16, 16, 16))
    with pytest.raises(ValueError, match="trajectory shape"):
        js.estimate_sensitivity_maps(k, np.zeros((8, 9, 3)), np.ones((8, 10)), image_shape_zyx=(16, 16, 16))
    with pytest.raises(ValueError, match="density shape"):
        js.estimate_sensitivity_maps(k, np.zeros((8, 10, 3)), np.ones((8, 9)), image_shape_zyx=(16, 16, 16))
