"""TVMW PDHG reconstruction on one GPU (b200 backend); CLI-compatible with the reference's ``algorithms/tvmw.py``."""

from ._common import TvmwReconstructor as _R, main_for

TvmwReconstructor = _R


def main(argv=None) -> int:
    return main_for("tvmw", argv)


if __name__ == "__main__":
    raise SystemExit(main())
