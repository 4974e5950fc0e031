"""Generate the observables and lattice-file fixtures of tests/golden/ from the
reference itself.

Runs the reference's own CondensateSigmaPi (observables.c:323) and
WriteBinaryLattice (simulation.c:129), compiled in place from the reference
tree by oracle/build_ref.py and driven through oracle/ref_harness.c, on seeded
sigma fields:
  golden_L{L}_sigma_obs.npz   sigma and the 8 CondensateSigmaPi outputs, L = 4, 8
                              (sigma centred on 0 and shifted to a mean of 0.3)
  golden_L4_lattice.bin       the reference's lattice file of a seeded sigma
  golden_L4_lattice.npz       that sigma, its sigmamass and the counters written

Only this script needs the reference tree; the fixtures travel without it.
Usage: python tests/golden/make_observables.py
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle.oracle import Ref  # noqa: E402

BETA_S = 0.85
NFLAV = 4
COUNTERS = dict(epsilon_link=0.0125, epsilon_pi=0.03, story_link=-3, story_sigma=7, story_pi=-2, accepted_link=11,
                done_link=13, accepted_sigma=95, done_sigma=100, accepted_pi=4, done_pi=9, measure=42)


def main():
    for L in (4, 8):
        ref = Ref(L)
        ref.init(1231, BETA_S, 0.2, 2)
        rng = np.random.default_rng(900 + L)
        V = L ** 3
        out = {}
        for name, shift in (("centred", 0.0), ("shifted", 0.3)):
            sigma = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V) + shift
            ref.set_sigma(sigma)
            out[f"sigma_{name}"] = sigma
            out[f"obs_{name}"] = ref.condensate_sigma()
        np.savez(HERE / f"golden_L{L}_sigma_obs.npz", **out)
        print(HERE / f"golden_L{L}_sigma_obs.npz")
        if L == 4:
            sigma = rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), V)
            ref.set_sigma(sigma)
            with tempfile.TemporaryDirectory() as d:
                path, copy = Path(d) / "terma.bin", Path(d) / "terma_copy.bin"
                ref.write_lattice(path, copy, COUNTERS)
                (HERE / "golden_L4_lattice.bin").write_bytes(path.read_bytes())
            np.savez(HERE / "golden_L4_lattice.npz", sigma=sigma, sigmamass=ref.sigmamass(),
                     counters=np.array([COUNTERS[k] for k in sorted(COUNTERS)], dtype=np.float64),
                     counter_names=np.array(sorted(COUNTERS)))
            print(HERE / "golden_L4_lattice.bin")


if __name__ == "__main__":
    main()
