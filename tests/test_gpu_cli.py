"""End-to-end CLI on the GPU: files in, CFL + manifest out, image vs the oracle."""

import json

import numpy as np
import pytest

from _dataset import write_dataset
from _fixtures import pkg
from oracle import nufft as onf
from oracle import pdhg as op

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("alg", ["tvm", "tvme", "tvmw"])
def test_reconstruct_cli_matches_oracle(tmp_path, alg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    write_dataset(tmp_path, shape=(24, 24, 22) if alg == "tvmw" else (16, 20, 24))
    cli = pkg("cli")
    out = tmp_path / "out"
    rc = cli.main(["reconstruct", "--algorithm", alg, "--", "--frac", "1.0", "--num-bins", "3", "--max-iter", "3",
                   "--tol", "0", "--output-dir", str(out), str(tmp_path), "img"])
    assert rc == 0
    cfl = pkg("cfl")
    E = 2
    img = cfl.read(out / f"img_e0-{E - 1}_m0-2")
    man = json.loads((out / "run_manifest.json").read_text())
    assert man["algorithm"] == alg and man["nufft_backend"] == "b200" and man["b200"]["iterations"] == 3
    common = pkg("algorithms._common")
    args = common.build_parser(alg).parse_args(["--frac", "1.0", "--num-bins", "3", str(tmp_path), "img"])
    prep = common.prepare(args, alg)
    coords, dcfs, ksps = [], [], []
    for b in range(3):
        idx = (prep.resp >= prep.bin_edges[b]) & (prep.resp < prep.bin_edges[b + 1])
        coords.append(prep.coord[idx]); dcfs.append(prep.dcf[idx]); ksps.append(prep.ksp[:, :, idx])
    pb = op.Problem(op.OracleNufft(prep.img_shape, coords), [k.astype(np.complex128) for k in ksps], dcfs, prep.mps)
    ref = op.run(alg, pb, max_iter=3, tol=0.0)
    got = img[:, 0, 0, :, 0, 0]
    assert got.shape == ref.image.shape
    assert onf.rel_l2(got, ref.image) < 1e-3
