"""The host steps either side of the PDHG path: respiratory self-navigation and
shard stitching, against golden vectors made by the reference's own code
(tests/golden/make_golden_host.py), plus their error behaviour and the CLI."""

import json

import numpy as np
import pytest

from _fixtures import GOLDEN, pkg


def test_respiratory_signal_matches_reference_golden():
    resp = pkg("respiratory")
    with np.load(GOLDEN / "resp.npz") as z:
        for i in range(2):
            got = resp.estimate_respiratory_signal(z[f"ksp{i}"], float(z[f"tr{i}"]))
            ref = z[f"resp{i}"]
            assert got.dtype == np.float32 and got.shape == ref.shape
            assert np.max(np.abs(got - ref)) < 1e-5, i
            assert got.min() == 0.0 and got.max() == 1.0


def test_respiratory_signal_single_echo_and_errors():
    resp = pkg("respiratory")
    with np.load(GOLDEN / "resp.npz") as z:
        ksp = z["ksp0"][:1]
        tr = float(z["tr0"])
    one = resp.estimate_respiratory_signal(ksp, tr)
    assert one.shape == (ksp.shape[2],)
    with pytest.raises(ValueError):
        resp.estimate_respiratory_signal(ksp[0], tr)                       # not 4-D
    with pytest.raises(ValueError):
        resp.estimate_respiratory_signal(ksp, 0.0)                         # TR
    with pytest.raises(ValueError):
        resp.estimate_respiratory_signal(ksp, 0.3)                         # 2 Hz cut above the 1.67 Hz Nyquist
    with pytest.raises(ValueError):
        resp.estimate_respiratory_signal(ksp, tr, config=resp.RespiratoryConfig(low_cut_hz=0.0))
    with pytest.raises(ValueError):
        resp.estimate_respiratory_signal(ksp, tr, config=resp.RespiratoryConfig(low_cut_hz=3.0, high_cut_hz=2.0))
    flat = np.ones((1, 2, 400, 1), dtype=np.complex64)
    with pytest.raises(ValueError, match="flat"):
        resp.estimate_respiratory_signal(flat, tr)


def _write_run(root, full, bins, echoes, stem="img", **man_over):
    cfl = pkg("cfl")
    for b0, b1 in bins:
        for e0, e1 in echoes:
            cfl.write(root / f"{stem}_e{e0}-{e1}_m{b0}-{b1}", full[b0:b1 + 1, :, :, e0:e1 + 1])
    man = {"output_stem": stem, "parameters": {"num_bins": full.shape[0], "num_echoes": full.shape[3]},
           "distributed": {"motion_groups": len(bins), "echo_groups": len(echoes)}}
    man.update(man_over)
    (root / "run_manifest.json").write_text(json.dumps(man), encoding="utf-8")


def test_stitch_matches_reference_golden(tmp_path):
    st, cfl = pkg("stitch"), pkg("cfl")
    with np.load(GOLDEN / "stitch.npz") as z:
        image = z["image"]
        bins = [tuple(int(v) for v in b) for b in z["bins"]]
        echoes = [tuple(int(v) for v in e) for e in z["echoes"]]
    _write_run(tmp_path, image, bins, echoes)
    base = st.stitch(tmp_path)
    assert base == (tmp_path / "imout").resolve()
    out = cfl.read(base)
    assert out.shape == image.shape and np.array_equal(out, image)
    with pytest.raises(FileExistsError):
        st.stitch(tmp_path)
    st.stitch(tmp_path, overwrite=True, output=tmp_path / "sub" / "again.cfl")
    assert np.array_equal(cfl.read(tmp_path / "sub" / "again"), image)


def test_stitch_rejects_bad_grids(tmp_path):
    st = pkg("stitch")
    rng = np.random.default_rng(0)
    full = rng.standard_normal((4, 1, 1, 3, 1, 1, 2, 3, 4)).astype(np.complex64)
    gap = tmp_path / "gap"
    gap.mkdir()
    _write_run(gap, full, [(0, 1), (3, 3)], [(0, 2)])
    with pytest.raises(ValueError, match="gap or overlap"):
        st.stitch(gap)
    missing = tmp_path / "missing"
    missing.mkdir()
    _write_run(missing, full, [(0, 1), (2, 3)], [(0, 0), (1, 2)])
    (missing / "img_e1-2_m2-3.hdr").unlink()
    (missing / "img_e1-2_m2-3.cfl").unlink()
    with pytest.raises(ValueError):
        st.stitch(missing)
    with pytest.raises(FileNotFoundError):
        st.stitch(tmp_path / "nowhere")
    good = tmp_path / "good"
    good.mkdir()
    _write_run(good, full, [(0, 3)], [(0, 2)])
    with pytest.raises(ValueError, match="file name"):
        st.stitch(good, output_name="a/b")
    with pytest.raises(ValueError, match="overwrite one of the shards"):
        st.stitch(good, output=good / "img_e0-2_m0-3.cfl")


def test_cli_resp_and_stitch(tmp_path, capsys):
    cli, cfl = pkg("cli"), pkg("cfl")
    with np.load(GOLDEN / "resp.npz") as z:
        ksp, tr, ref = z["ksp0"], float(z["tr0"]), z["resp0"]
    raw = tmp_path / "raw"
    raw.mkdir()
    E, C, T, R = ksp.shape
    cfl.write(raw / "ksp", ksp.reshape(1, 1, 1, E, 1, C, T, R, 1))
    (raw / "tr.txt").write_text(f"{tr}\n", encoding="utf-8")
    assert cli.main(["resp", str(raw), "--work-dir", str(tmp_path / "work")]) == 0
    got = cfl.read(tmp_path / "work" / "resp")
    assert got.shape == (T, 1) and np.max(np.abs(got[:, 0].real - ref)) < 1e-5
    with np.load(GOLDEN / "stitch.npz") as z:
        image = z["image"]
        bins = [tuple(int(v) for v in b) for b in z["bins"]]
        echoes = [tuple(int(v) for v in e) for e in z["echoes"]]
    run = tmp_path / "run"
    run.mkdir()
    _write_run(run, image, bins, echoes)
    assert cli.main(["stitch", str(run), "--output-name", "whole"]) == 0
    assert np.array_equal(cfl.read(run / "whole"), image)
    assert "Wrote" in capsys.readouterr().out
