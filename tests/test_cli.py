"""Single-rank problem assembly of the CLI against the reference's preparation rules (CPU)."""

import argparse

import numpy as np
import pytest

from _dataset import write_dataset
from _fixtures import pkg


def _args(alg, root, **kw):
    common = pkg("algorithms._common")
    argv = [str(root), "out"] + [x for k, v in kw.items() for x in (k, str(v))]
    return common.build_parser(alg).parse_args(argv)


@pytest.mark.parametrize("alg", ["tvm", "tvme", "tvmw"])
def test_prepare_follows_reference_rules(tmp_path, alg):
    ds = write_dataset(tmp_path)
    common = pkg("algorithms._common")
    args = _args(alg, tmp_path, **{"--frac": 1.0, "--num-bins": 3})
    prep = common.prepare(args, alg)
    TR = ds.coord.shape[0]
    # trajectories kept: TVM / TVME drop the 2 % respiratory outliers, TVMW keeps all
    keep = np.arange(TR)
    if alg != "tvmw":
        lo, hi = np.percentile(ds.resp, 2), np.percentile(ds.resp, 98)
        keep = keep[(ds.resp > lo) & (ds.resp < hi)]
    resp = ds.resp[keep]
    edges = np.percentile(resp, np.linspace(0, 100, 4))
    np.testing.assert_allclose(prep.bin_edges, edges)
    sel = np.zeros(resp.shape, bool)
    for b in range(3):
        sel |= (resp >= edges[b]) & (resp < edges[b + 1])
    idx = keep[sel]
    assert prep.ksp.shape == (2, 3, idx.size, ds.coord.shape[1])
    np.testing.assert_allclose(prep.coord, ds.coord[idx], rtol=1e-5, atol=1e-4)   # physical -> grid units
    assert abs(float(np.abs(prep.ksp).max()) - 1.0) < 1e-6                      # ksp / max |ksp|
    np.testing.assert_allclose(np.sqrt((np.abs(prep.mps) ** 2).sum(0)), 1.0, rtol=1e-5)
    assert abs(float(prep.dcf.max()) - 1.0) < 1e-6                               # dcf / max
    assert prep.img_shape == ds.cfg.img_shape


def test_rejects_node_grid(tmp_path):
    write_dataset(tmp_path)
    common = pkg("algorithms._common")
    args = _args("tvme", tmp_path, **{"--echo-groups": 2})
    with pytest.raises(ValueError, match="one device"):
        common.prepare(args, "tvme")


def test_cli_dispatch_parses_forwarded_arguments():
    cli = pkg("cli")
    a = cli.build_parser().parse_args(["reconstruct", "--algorithm", "tvmw", "--", "--lambda2", "1e-4", "in", "o"])
    assert a.algorithm == "tvmw" and a.algorithm_arguments[1:] == ["--lambda2", "1e-4", "in", "o"]


def test_cfl_roundtrip(tmp_path):
    cfl = pkg("cfl")
    a = (np.arange(24).reshape(2, 3, 4) * (1 + 0.5j)).astype(np.complex64)
    cfl.write(tmp_path / "x", a)
    hdr = (tmp_path / "x.hdr").read_text().splitlines()[1].split()
    assert hdr == ["4", "3", "2"]                     # reversed dimensions, C-order payload
    np.testing.assert_array_equal(cfl.read(tmp_path / "x"), a)
