"""CPU tests of the C-ABI boundary: the libraries load, export every function
their headers declare, and fail loudly (no CPU fallback) without a GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
INCLUDE = ROOT / "include"
LIBDIR = ROOT / "3d-gross-neveu-model_b200" / "lib"


def declared(header: str):
    """Function names declared with GN_API in include/<header>."""
    text = "\n".join(ln for ln in (INCLUDE / header).read_text().splitlines() if not ln.startswith("#"))
    return sorted(set(re.findall(r"GN_API[^;(]*?\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)))


def exported(lib: Path):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


@pytest.fixture(scope="module")
def core_lib():
    import gn_b200
    gn_b200.load_library()
    return gn_b200.LIB_PATH


def test_core_exports_every_declared_symbol(core_lib):
    names = declared("gn_b200.h")
    assert len(names) >= 18
    missing = set(names) - exported(core_lib)
    assert not missing, missing


def test_core_loads_and_fails_loudly_without_gpu(core_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import gn_b200
    with pytest.raises(gn_b200.GnError) as e:
        gn_b200.Lattice(8)
    assert e.value.status == -5  # GN_ERR_NO_DEVICE


def test_bad_lattice_size_rejected(core_lib):
    import gn_b200
    lib = gn_b200.load_library()
    ctx = C.c_void_p()
    assert lib.gn_create(C.byref(ctx), 7, 0) != 0  # odd L: the fermion order needs even L
    assert not ctx.value


def test_dropin_exports_every_declared_symbol(core_lib):
    lib = LIBDIR / "libgn_dropin.so"
    assert lib.exists(), "build the library first (python 3d-gross-neveu-model_b200/build.py)"
    names = declared("gn_dropin.h")
    assert len(names) >= 21
    missing = set(names) - exported(lib)
    assert not missing, missing


def test_dropin_pi_exports_every_declared_symbol(core_lib):
    """The PI_INTERACTION layer exports every function of gn_dropin.h (with
    the complex M) and gn_dropin_pi.h's."""
    lib = LIBDIR / "libgn_dropin_pi.so"
    assert lib.exists(), "build the library first (python 3d-gross-neveu-model_b200/build.py)"
    names = set(declared("gn_dropin.h")) | set(declared("gn_dropin_pi.h"))
    assert len(names) >= 30
    missing = names - exported(lib)
    assert not missing, missing


def test_dropin_struct_layout_matches_reference(tmp_path):
    """The drop-in restates the reference's structs; their sizes and member
    offsets must equal the reference build's (recorded by
    tests/golden/make_golden.py from the reference's own headers)."""
    import subprocess

    import numpy as np
    exe = tmp_path / "layout_probe"
    subprocess.run(["gcc", "-std=gnu11", f"-I{INCLUDE}", str(ROOT / "tests" / "golden" / "layout_probe.c"), "-o",
                    str(exe)], check=True)
    got = np.array([int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
                    .split()])
    ref = np.load(ROOT / "tests" / "golden" / "layout_reference.npy")
    assert np.array_equal(got, ref), (got, ref)
