"""The exact-order mode's |z| (csrc/host_hypot.h) reproduces the host C
library's hypot bit for bit, and the library's pow(a, 2.0) is a * a: the two
operations conjugategradient.c:65 applies to every complex site."""
import subprocess

from conftest import ROOT


def test_host_hypot_matches_libm(tmp_path):
    exe = tmp_path / "host_hypot_check"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-I", str(ROOT / "3d-gross-neveu-model_b200" / "csrc"),
                    str(ROOT / "tests" / "host_hypot_check.c"), "-o", str(exe), "-lm"], check=True)
    out = subprocess.run([str(exe), "4000000"], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["0", "0"], out
