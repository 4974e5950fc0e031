"""The row items every sweep of the Dirac and solver kernels visits
(csrc/rowvec.cuh) reproduce the one-site geometry exactly: checked on the host
for every site at L = 4 .. 256 and every item width."""
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not found")
def test_item_geometry(tmp_path):
    exe = tmp_path / "item_geometry_check"
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", str(ROOT / "3d-gross-neveu-model_b200" / "csrc"),
                    str(ROOT / "tests" / "item_geometry_check.cu"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "total bad 0" in r.stdout
