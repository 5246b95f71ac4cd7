"""b200 JSENSE against the CPU restatement (oracle/jsense.py) on one phantom."""

import numpy as np
import pytest

from _fixtures import pkg
from oracle import jsense as oj
from test_jsense_cpu import _problem, rss

pytestmark = pytest.mark.gpu


def test_b200_jsense_matches_oracle_and_recovers_maps():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    js = pkg("jsense")
    coord, dcf, mps, img, y = _problem(shape=(32, 32, 32), cones=256, readout=200)
    kw = dict(ker_width=8, calib_width=16, max_iter=3, inner=5)
    got = js.jsense_calibration(y, coord, dcf, device=0, **kw).cpu().numpy()
    ref = oj.jsense(y, coord, dcf, **kw)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < 1e-3, err
    full = js.estimate_sensitivity_maps(
        y.reshape(1, 4, 256, 200).astype(np.complex64), coord.reshape(256, 200, 3), dcf.reshape(256, 200),
        image_shape_zyx=img.shape, config=js.JsenseConfig(mps_kernel_width=8, kspace_calibration_width=16,
                                                          max_iter=3, max_inner_iter=5))
    assert full.shape == (4,) + img.shape and full.dtype == np.complex64
    corr = np.abs(np.sum(np.conj(rss(full)) * rss(mps), 0))[img != 0]
    assert np.median(corr) > 0.99, np.median(corr)
