"""Assemble motion x echo reconstruction shards into one CFL image.

The reference's ``toporecon stitch`` (``src/toporecon/postprocessing/stitch.py:191-256``):
a reconstruction run writes one nine-dimensional CFL per (motion range, echo
range) tile, named ``<stem>_e<e0>-<e1>_m<b0>-<b1>`` (inclusive ranges), next
to ``run_manifest.json``, which records the grid (``parameters.num_bins``,
``parameters.num_echoes``, ``distributed.motion_groups`` / ``echo_groups``).
``stitch`` finds the tiles, checks that they cover the grid exactly once with
compatible shapes, and copies them into one (B, 1, 1, E, 1, 1, Z, Y, X) array
written atomically (a temporary file renamed into place).  The b200
reconstructor writes a single tile covering every bin and echo; multi-rank
runs write one per rank.  Host file work only.
"""

from __future__ import annotations

import json
import os
import re
import uuid
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import cfl as _cfl


@dataclass(frozen=True)
class Tile:
    base: Path
    echoes: tuple          # [e0, e1) half-open
    bins: tuple            # [b0, b1) half-open
    shape: tuple


def _manifest(directory: Path) -> dict:
    path = directory / "run_manifest.json"
    if not path.is_file():
        raise FileNotFoundError(f"{path}: no run manifest next to the shards")
    try:
        data = json.loads(path.read_text(encoding="utf-8"))
    except json.JSONDecodeError as exc:
        raise ValueError(f"{path}: not valid JSON ({exc})") from exc
    if not isinstance(data, dict):
        raise ValueError(f"{path}: the manifest is not a JSON object")
    return data


def _tiles(directory: Path, stem: str) -> list:
    rel = Path(stem)
    if rel.is_absolute() or not rel.name:
        raise ValueError(f"the shard prefix {stem!r} has to be a name relative to the run directory")
    folder = (directory / rel.parent).resolve()
    if folder != directory and directory not in folder.parents:
        raise ValueError(f"the shard prefix {stem!r} leaves the run directory")
    if not folder.is_dir():
        raise FileNotFoundError(f"{folder}: the shard directory does not exist")
    pat = re.compile(re.escape(rel.name) + r"_e(\d+)-(\d+)_m(\d+)-(\d+)\.hdr")
    out = []
    for hdr in sorted(folder.iterdir()):
        m = pat.fullmatch(hdr.name)
        if not m:
            continue
        base = hdr.with_suffix("")
        payload = base.with_suffix(".cfl")
        if not payload.is_file():
            raise FileNotFoundError(f"{payload}: the shard's payload is missing")
        shape = _cfl.read_header(base)
        need = int(np.prod(shape, dtype=np.int64)) * _cfl.CFL_DTYPE.itemsize
        if payload.stat().st_size != need:
            raise ValueError(f"{payload}: {payload.stat().st_size} bytes, its header needs {need}")
        e0, e1, b0, b1 = (int(g) for g in m.groups())
        out.append(Tile(base=base, echoes=(e0, e1 + 1), bins=(b0, b1 + 1), shape=tuple(shape)))
    if not out:
        raise FileNotFoundError(f"no shards named {rel.name}_e*-*_m*-* in {folder}")
    return out


def _covers(ranges: set, total: int, what: str) -> None:
    pos = 0
    for lo, hi in sorted(ranges):
        if lo != pos or hi <= lo:
            raise ValueError(f"the {what} ranges of the shards leave a gap or overlap at {what} {pos}")
        pos = hi
    if pos != total:
        raise ValueError(f"the {what} ranges of the shards end at {pos}, not at {total}")


def _check(tiles: list, man: dict) -> tuple:
    try:
        n_bins = int(man["parameters"]["num_bins"])
        mg = int(man["distributed"]["motion_groups"])
        eg = int(man["distributed"]["echo_groups"])
    except (KeyError, TypeError, ValueError) as exc:
        raise ValueError("the manifest lacks num_bins / motion_groups / echo_groups") from exc
    if min(n_bins, mg, eg) < 1:
        raise ValueError("num_bins, motion_groups and echo_groups have to be positive")
    if len(tiles) != mg * eg:
        raise ValueError(f"the manifest's {mg} x {eg} grid needs {mg * eg} shards; found {len(tiles)}")
    rec = man["parameters"].get("num_echoes")
    try:
        n_echoes = max(t.echoes[1] for t in tiles) if rec is None else int(rec)
    except (TypeError, ValueError) as exc:
        raise ValueError(f"the manifest's echo count {rec!r} is not an integer") from exc
    if n_echoes < 1:
        raise ValueError(f"the manifest's echo count {n_echoes} is not positive")
    bins = {t.bins for t in tiles}
    echoes = {t.echoes for t in tiles}
    if len(bins) != mg or len(echoes) != eg:
        raise ValueError("the shards' ranges do not form the manifest's motion x echo grid")
    if {(t.bins, t.echoes) for t in tiles} != {(b, e) for b in bins for e in echoes}:
        raise ValueError("a tile of the motion x echo grid is missing or repeated")
    _covers(bins, n_bins, "motion")
    _covers(echoes, n_echoes, "echo")
    ref = list(tiles[0].shape)
    if len(ref) != 9 or any(ref[a] != 1 for a in (1, 2, 4, 5)):
        raise ValueError(f"{tiles[0].base}: expected a (B, 1, 1, E, 1, 1, Z, Y, X) shard, got {tuple(ref)}")
    for t in tiles:
        if len(t.shape) != 9:
            raise ValueError(f"{t.base}: expected nine dimensions, got {t.shape}")
        if t.shape[0] != t.bins[1] - t.bins[0] or t.shape[3] != t.echoes[1] - t.echoes[0]:
            raise ValueError(f"{t.base}: its shape {t.shape} disagrees with the ranges in its name")
        if any(t.shape[a] != ref[a] for a in range(9) if a not in (0, 3)):
            raise ValueError(f"{t.base}: its shape {t.shape} does not match {tuple(ref)}")
    ref[0], ref[3] = n_bins, n_echoes
    return tuple(ref)


def _output_base(directory: Path, output_name: str, output) -> Path:
    if output is None:
        name = Path(output_name)
        if name.is_absolute() or len(name.parts) != 1 or output_name in (".", ".."):
            raise ValueError(f"--output-name {output_name!r} has to be a file name, not a path")
        target = directory / name
    else:
        target = Path(output).expanduser()
    if target.suffix not in ("", ".hdr", ".cfl"):
        raise ValueError(f"{target}: give a base path, or one ending in .hdr or .cfl")
    return _cfl.base_path(target).resolve()


def stitch(directory, *, stem: str | None = None, output_name: str = "imout", output=None,
           overwrite: bool = False) -> Path:
    """Assemble the shards of one run into ``<output>.hdr/.cfl``; returns the base path."""
    root = Path(directory).expanduser().resolve()
    if not root.is_dir():
        raise FileNotFoundError(f"{root}: the run directory does not exist")
    man = _manifest(root)
    stem = stem or man.get("output_stem")
    if not isinstance(stem, str) or not stem:
        raise ValueError("no shard prefix given and the manifest has no output_stem")
    tiles = _tiles(root, stem)
    shape = _check(tiles, man)
    base = _output_base(root, output_name, output)
    inputs = {p.resolve() for t in tiles for p in (t.base.with_suffix(".hdr"), t.base.with_suffix(".cfl"))}
    if base.with_suffix(".hdr") in inputs or base.with_suffix(".cfl") in inputs:
        raise ValueError(f"{base}: the output would overwrite one of the shards")
    if not overwrite and (base.with_suffix(".hdr").exists() or base.with_suffix(".cfl").exists()):
        raise FileExistsError(f"{base}: exists (pass overwrite=True to replace it)")
    base.parent.mkdir(parents=True, exist_ok=True)
    tmp = base.parent / f".stitch-{uuid.uuid4().hex}"
    try:
        dst = np.memmap(tmp.with_suffix(".cfl"), mode="w+", dtype=_cfl.CFL_DTYPE, shape=shape)
        for t in tiles:
            src = _cfl.read(t.base, mmap=True)
            dst[t.bins[0]:t.bins[1], :, :, t.echoes[0]:t.echoes[1]] = src
            del src
        dst.flush()
        del dst
        with tmp.with_suffix(".hdr").open("w", encoding="utf-8") as fh:
            fh.write("# Dimensions\n" + " ".join(str(d) for d in reversed(shape)) + "\n")
        os.replace(tmp.with_suffix(".cfl"), base.with_suffix(".cfl"))
        os.replace(tmp.with_suffix(".hdr"), base.with_suffix(".hdr"))
    finally:
        for suffix in (".cfl", ".hdr"):
            tmp.with_suffix(suffix).unlink(missing_ok=True)
    return base
