"""Build the in-tree CUDA library ``libtoporecon_b200.so`` for sm_100a.

    python multinodemri-miccai26_b200/build.py [--force] [--verbose]

nvcc compiles every ``csrc/*.cu`` for ``sm_100a`` only (no PTX for other
targets, no multi-architecture fat binary) and links one shared library next
to this file.  The library exports the C ABI declared in
``include/toporecon_b200.h``.  Rebuilds only when a source or header is newer
than the library.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = REPO / "include"
LIB = PKG / "libtoporecon_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-Xptxas", "-O3",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the b200 backend needs the CUDA 12.9 toolkit to build")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(sources()) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    if not force and not needs_build():
        return LIB
    nvcc = nvcc_path()
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    cmds, objs = [], []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmds.append([nvcc, *NVCC_FLAGS, *(extra or []), f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)])
        objs.append(str(obj))
    # one nvcc per translation unit, in parallel (the largest unit sets the build time)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd), flush=True)
        for f in [ex.submit(subprocess.run, cmd, check=True) for cmd in cmds]:
            f.result()
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    args = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if args.ptxas_verbose else None
    path = build(force=args.force or args.ptxas_verbose, verbose=args.verbose, extra=extra)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
