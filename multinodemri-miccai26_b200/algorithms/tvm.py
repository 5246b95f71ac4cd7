"""TVM PDHG reconstruction on one GPU (b200 backend); CLI-compatible with the reference's ``algorithms/tvm.py``."""

from ._common import TvmReconstructor as _R, main_for

TvmReconstructor = _R


def main(argv=None) -> int:
    return main_for("tvm", argv)


if __name__ == "__main__":
    raise SystemExit(main())
