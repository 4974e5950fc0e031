"""The batched chains' Philox4x64-10 (csrc/philox.cuh, built here for the
host from the same source as the device code) equals numpy.random.Philox,
an independent implementation of the published generator, block for block."""
import subprocess

import numpy as np

from conftest import ROOT


def test_philox_matches_numpy(tmp_path):
    exe = tmp_path / "philox_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "3d-gross-neveu-model_b200" / "csrc"),
                    str(ROOT / "tests" / "philox_check.cpp"), "-o", str(exe)], check=True)
    rng = np.random.default_rng(7)
    cases = []
    for _ in range(40):
        key = [int(x) for x in rng.integers(0, 2 ** 63, size=2)]
        ctr = [int(x) for x in rng.integers(0, 2 ** 63, size=4)]
        cases.append((key, ctr))
    cases.append(([0, 0], [0, 0, 0, 0]))
    cases.append(([2 ** 64 - 1] * 2, [2 ** 64 - 1] * 4))
    inp = "".join("%x %x %x %x %x %x\n" % (k[0], k[1], *c) for k, c in cases)
    out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    for (key, ctr), line in zip(cases, out):
        # numpy increments its 256-bit counter before each block: start one below
        c = sum(v << (64 * i) for i, v in enumerate(ctr))
        c = (c - 1) % (1 << 256)
        g = np.random.Philox(key=key, counter=[(c >> (64 * i)) & (2 ** 64 - 1) for i in range(4)])
        want = ["%016x" % int(v) for v in g.random_raw(4)]
        assert line.split() == want, (key, ctr)
