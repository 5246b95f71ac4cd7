"""TVME PDHG reconstruction on one GPU (b200 backend); CLI-compatible with the reference's ``algorithms/tvme.py``."""

from ._common import TvmeReconstructor as _R, main_for

TvmeReconstructor = _R


def main(argv=None) -> int:
    return main_for("tvme", argv)


if __name__ == "__main__":
    raise SystemExit(main())
