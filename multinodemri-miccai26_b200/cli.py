"""``toporecon reconstruct`` front-end for the b200 backend.

    python -m multinodemri-miccai26_b200 reconstruct --algorithm tvme -- [reference tvme flags] input_dir img_file

Mirrors the reference's dispatch (``src/toporecon/cli.py:149-164``): the
arguments after ``--`` go to the algorithm's ``main``.  Only ``reconstruct``
belongs to the accelerated path; of the reference's other sub-commands
(inspect, resp, jsense, prepare, stitch) only the JSENSE estimation exists
here, as the library function ``jsense.estimate_sensitivity_maps``.
"""

from __future__ import annotations

import argparse
import importlib
import logging
import sys


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="toporecon-b200")
    p.add_argument("--verbose", action="store_true")
    sub = p.add_subparsers(dest="command", required=True)
    rec = sub.add_parser("reconstruct", help="run TVM / TVME / TVMW PDHG on one GPU")
    rec.add_argument("--algorithm", choices=("tvm", "tvme", "tvmw"), required=True)
    rec.add_argument("algorithm_arguments", nargs=argparse.REMAINDER)
    return p


def main(argv=None) -> int:
    args = build_parser().parse_args(argv)
    logging.basicConfig(level=logging.DEBUG if args.verbose else logging.INFO, format="%(levelname)s: %(message)s")
    forwarded = list(args.algorithm_arguments)
    if forwarded[:1] == ["--"]:
        forwarded = forwarded[1:]
    pkg = __name__.rsplit(".", 1)[0]
    mod = importlib.import_module(f"{pkg}.algorithms.{args.algorithm}")
    return mod.main(forwarded)


if __name__ == "__main__":
    sys.exit(main())
