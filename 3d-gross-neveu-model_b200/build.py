"""Build recipe of the CUDA library (sm_100a only).

Compiles csrc/*.cu with nvcc into lib/libgn_b200.so (the C-ABI of
include/gn_b200.h) and csrc/dropin.cpp into lib/libgn_dropin.so (the
reference-signature layer of include/gn_dropin.h) and, with GN_DROPIN_PI, into
lib/libgn_dropin_pi.so (the same layer for the PI_INTERACTION build,
include/gn_dropin_pi.h).  The FP64 translation unit
engine.cu is compiled with --fmad=false so that the FP64 kernels round like the
reference's x86-64 build (multiply, then add).

Usage: python build.py [--force] [--verbose]   (``-Xptxas -v`` with --verbose)
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = PKG.parent / "include"
OBJ = LIB / "obj"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              f"-I{INCLUDE}"]
UNITS = {
    "engine.cu": ["--fmad=false"],
    "mixed.cu": [],
    "capi.cu": [],
    "noalloc.cu": ["--fmad=false"],
    "exact.cu": ["--fmad=false"],
    "ensemble.cu": ["--fmad=false"],
    "serve.cu": ["--fmad=false"],
    "checkpoint.cu": [],
    "u1.cu": ["--fmad=false"],
    "selftest.cu": [],
}
CORE_LIB = LIB / "libgn_b200.so"
DROPIN_LIB = LIB / "libgn_dropin.so"
DROPIN_PI_LIB = LIB / "libgn_dropin_pi.so"  # the same source with GN_DROPIN_PI: the U(1) (PI_INTERACTION) build


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    return "nvcc"


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    LIB.mkdir(exist_ok=True)
    OBJ.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    objs = []
    procs = []
    for unit, extra in UNITS.items():
        src = CSRC / unit
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, Path(__file__), *headers]):
            cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append((unit, subprocess.Popen(cmd)))
    for unit, p in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {unit}")
    if force or _stale(CORE_LIB, objs):
        subprocess.run([_nvcc(), *ARCH, "-shared", "-o", str(CORE_LIB), *map(str, objs), "-lcudart"], check=True)
    dropin = CSRC / "dropin.cpp"
    for lib, defs in ((DROPIN_LIB, []), (DROPIN_PI_LIB, ["-DGN_DROPIN_PI"])):
        if dropin.exists() and (force or _stale(lib, [dropin, CORE_LIB, *headers])):
            subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", *defs, f"-I{INCLUDE}", "-o",
                            str(lib), str(dropin), f"-L{LIB}", "-lgn_b200", "-Wl,-rpath,$ORIGIN", "-ldl"], check=True)
    return CORE_LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
