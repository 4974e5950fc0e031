"""Build recipe for the reference oracle -- TEST INFRASTRUCTURE.

Compiles the reference's own C sources where they lie (the reference tree,
read-only) together with oracle/ref_harness.c into one shared object per
lattice size, written only to oracle/_ref/.  No reference source is copied:
oracle/ref_config.h is pre-included with ``gcc -include`` and supplies the
configuration of macro.h (with a variable LSPACE), so the reference's own
macro.h body is skipped by its include guard.

Flags follow the reference README's build line (``gcc -O3 *.c -lm``), plus
``-fcommon`` (new_random.h:22 defines ``random_state`` in a header that two
files include) and ``-fPIC -shared`` so ctypes can load the result.  test.c
(the reference ``main``) is left out; the harness replaces it.

The reference tree is taken from --reference DIR, else from the environment
variable GN_REFERENCE_DIR, else from a directory named "reference" beside the
repository's own directory.  Without it nothing is built, and the objects
already under oracle/_ref/ are used as they are.

Usage:  python oracle/build_ref.py [--reference DIR] [--L 4 8 16 ...] [--integrator 0 1 2]
Outputs: oracle/_ref/libgnref_L{L}_i{I}{tag}.so
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF_DIR = Path(os.environ.get("GN_REFERENCE_DIR") or HERE.parent.parent / "reference")

DEFAULT_L = (4, 6, 8, 12, 16, 24, 32, 48, 64)
PI_DEFS, PI_TAG = ("-DPI_INTERACTION",), "_pi"  # the U(1) model's build
# every CG stopped at 1e-10 |phi| (ref_config.h): the benchmark's CPU arm
REL_DEFS, REL_TAG = ("-DGN_REF_RELATIVE_TOL=1e-10",), "_rel"
CFLAGS = ["-O3", "-fcommon", "-fPIC", "-w"]


def reference_sources() -> list[Path]:
    return sorted(p for p in REF_DIR.glob("*.c") if p.name != "test.c")


def lib_path(L: int, integrator: int = 0, tag: str = "") -> Path:
    return OUT / f"libgnref_L{L}_i{integrator}{tag}.so"


def available() -> bool:
    return REF_DIR.is_dir() and (REF_DIR / "dirac.c").is_file()


def _compile(src: Path, obj: Path, defs: list[str]) -> None:
    cmd = ["gcc", *CFLAGS, *defs, "-include", str(HERE / "ref_config.h"), f"-I{REF_DIR}", "-c", str(src), "-o",
           str(obj)]
    subprocess.run(cmd, check=True)


def build(L: int, integrator: int = 0, extra_defs: tuple[str, ...] = (), tag: str = "", force: bool = False) -> Path:
    """Compile the reference at lattice size L; return the shared object path."""
    if not available():
        raise FileNotFoundError(f"reference sources not found under {REF_DIR}")
    if L % 2 or L < 2:
        raise ValueError("the fermion ordering of the reference needs an even L >= 2")
    out = lib_path(L, integrator, tag)
    srcs = reference_sources() + [HERE / "ref_harness.c"]
    deps = srcs + [HERE / "ref_config.h", Path(__file__)]
    if out.exists() and not force and out.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return out
    objdir = OUT / f"obj_L{L}_i{integrator}{tag}"
    objdir.mkdir(parents=True, exist_ok=True)
    defs = [f"-DGN_REF_L={L}", f"-DGN_REF_INTEGRATOR={integrator}", *extra_defs]
    objs = [objdir / (s.stem + ".o") for s in srcs]
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        list(ex.map(lambda so: _compile(so[0], so[1], defs), zip(srcs, objs)))
    subprocess.run(["gcc", "-shared", "-o", str(out), *map(str, objs), "-lm"], check=True)
    return out


def build_all(Ls=DEFAULT_L, integrators=(0,)) -> list[Path]:
    OUT.mkdir(parents=True, exist_ok=True)
    built = []
    for L in Ls:
        for i in integrators:
            built.append(build(L, i))
    # alternative integrators are pinned at the small sizes only
    for L in (4, 8):
        for i in (1, 2):
            built.append(build(L, i))
    # the U(1) model (PI_INTERACTION): the test sizes and the benchmark's L = 64
    for L in (4, 8, 64):
        built.append(build(L, 0, PI_DEFS, PI_TAG))
    # every solve to 1e-10 |phi|: the benchmark's workload (L = 64) for the CPU
    # baseline, and L = 8 for the test of the reference arm
    for L in (8, 64):
        built.append(build(L, 0, REL_DEFS, REL_TAG))
    return built


def main() -> int:
    global REF_DIR
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="the reference's source tree")
    ap.add_argument("--L", type=int, nargs="*", default=list(DEFAULT_L))
    ap.add_argument("--integrator", type=int, nargs="*", default=[0])
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    if a.reference:
        REF_DIR = Path(a.reference)
    if not available():
        print(f"reference not present at {REF_DIR}; nothing to build", file=sys.stderr)
        return 0
    OUT.mkdir(parents=True, exist_ok=True)
    for L in a.L:
        for i in a.integrator:
            print(build(L, i, force=a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
