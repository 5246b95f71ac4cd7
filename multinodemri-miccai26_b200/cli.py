"""``toporecon reconstruct`` front-end for the b200 backend.

    python -m multinodemri-miccai26_b200 reconstruct --algorithm tvme -- [reference tvme flags] input_dir img_file

Mirrors the reference's dispatch (``src/toporecon/cli.py:149-164``): the
arguments after ``--`` go to the algorithm's ``main``.  ``reconstruct`` is the
accelerated path; ``resp`` (respiratory self-navigation, ``cli.py:74-79``,
``:190-193``) and ``stitch`` (shard assembly, ``cli.py:107-127``, ``:173-183``)
are the host steps either side of it, with the reference's arguments.  The
reference's ``inspect`` / ``jsense`` / ``prepare`` commands are not
sub-commands here; the JSENSE estimation itself is the library function
``jsense.estimate_sensitivity_maps``.
"""

from __future__ import annotations

import argparse
import importlib
import logging
import sys
from pathlib import Path


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="toporecon-b200")
    p.add_argument("--verbose", action="store_true")
    sub = p.add_subparsers(dest="command", required=True)
    rec = sub.add_parser("reconstruct", help="run TVM / TVME / TVMW PDHG on one GPU")
    rec.add_argument("--algorithm", choices=("tvm", "tvme", "tvmw"), required=True)
    rec.add_argument("algorithm_arguments", nargs=argparse.REMAINDER)
    resp = sub.add_parser("resp", help="estimate resp.hdr/.cfl from a raw dataset into a work directory")
    resp.add_argument("input", type=Path)
    resp.add_argument("--work-dir", type=Path, required=True)
    st = sub.add_parser("stitch", help="assemble the reconstruction shards of a run into one CFL image")
    st.add_argument("input_dir", type=Path)
    st.add_argument("--input-prefix", "--stem", dest="stem", help="shard prefix (default: the manifest's output_stem)")
    out = st.add_mutually_exclusive_group()
    out.add_argument("--output-name", default="imout", help="file name of the image inside INPUT_DIR")
    out.add_argument("--output", type=Path, help="full path of the image")
    st.add_argument("--overwrite", action="store_true")
    return p


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    logging.basicConfig(level=logging.DEBUG if args.verbose else logging.INFO, format="%(levelname)s: %(message)s")
    pkg = __name__.rsplit(".", 1)[0]
    if args.command == "resp":
        args.work_dir.mkdir(parents=True, exist_ok=True)
        out = importlib.import_module(f"{pkg}.respiratory").estimate_respiratory_from_dataset(args.input,
                                                                                               args.work_dir)
        print(f"Wrote {out}.hdr and {out}.cfl")
        return 0
    if args.command == "stitch":
        out = importlib.import_module(f"{pkg}.stitch").stitch(args.input_dir, stem=args.stem,
                                                              output_name=args.output_name, output=args.output,
                                                              overwrite=args.overwrite)
        print(f"Wrote {out}.hdr and {out}.cfl")
        return 0
    forwarded = list(args.algorithm_arguments)
    if forwarded[:1] == ["--"]:
        forwarded = forwarded[1:]
    mod = importlib.import_module(f"{pkg}.algorithms.{args.algorithm}")
    return mod.main(forwarded)


if __name__ == "__main__":
    sys.exit(main())
