"""Build recipe of libnozomi_b200.so (in-tree, sm_100a).

    python -m nozomi_b200.build [--force] [--verbose]

Every .cu under nozomi_b200/csrc is compiled with nvcc for sm_100a only, with
--fmad=false (no implicit multiply-add contraction: expressions round in source
order, the precondition of bit-exact parity with the reference's arithmetic)
and linked into nozomi_b200/libnozomi_b200.so with the static CUDA runtime.
With --debug the same sources are built with -DNZ_DEBUG_BOUNDS=1 into
libnozomi_b200_debug.so, the bounds-checked variant.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libnozomi_b200.so"
BUILD_DIR = PKG / "_build"
# the bounds-checked build (-DNZ_DEBUG_BOUNDS=1): loaded when
# NOZOMI_B200_DEBUG_BOUNDS=1, for tests and debugging
DEBUG_LIB = PKG / "libnozomi_b200_debug.so"
DEBUG_BUILD_DIR = PKG / "_build_debug"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
              "--expt-relaxed-constexpr", "-I", str(INCLUDE), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def _deps():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def build(force: bool = False, verbose: bool = False, extra=None, debug: bool = False) -> Path:
    """Build the library (debug: the bounds-checked variant beside it)."""
    lib, bdir = (DEBUG_LIB, DEBUG_BUILD_DIR) if debug else (LIB, BUILD_DIR)
    if not force and not stale(lib):
        return lib
    bdir.mkdir(exist_ok=True)
    objs = []
    flags = NVCC_FLAGS + (["-DNZ_DEBUG_BOUNDS=1"] if debug else [])
    for src in sources():
        obj = bdir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *flags, *(extra or []), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = str(lib) + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    ap.add_argument("--debug", action="store_true", help="the bounds-checked variant (libnozomi_b200_debug.so)")
    a = ap.parse_args(argv)
    extra = ["-Xptxas", "-v"] if a.ptxas_info else None
    print(build(force=a.force or a.ptxas_info, verbose=a.verbose, extra=extra, debug=a.debug))


if __name__ == "__main__":
    sys.exit(main())
