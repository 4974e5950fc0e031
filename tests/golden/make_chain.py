"""Generate tests/golden/golden_L8_chains.npz: the reference's own chains of
LeapFrog2MinimumNormSigmaVelocityFirst trajectories at L = 8, beta_s = 0.85,
dSFMT seed 1231:
  - "readme": 1000 trajectories at the README configuration (eps = 0.2,
    2 steps), where |dH| < 0.01 and every trajectory is accepted;
  - "reject": 500 trajectories at eps = 1.0, 2 steps, where about a quarter are
    rejected, so the restore-on-reject path runs inside the chain.

The reference (oracle/build_ref.py, driven through oracle/ref_harness.c) runs
the chain from a seeded sigma ~ N(0, 2/(N_f beta_s)) and its acceptance file
gives dH with 16 decimals (moleculardynamics.c:1426).  The fixture keeps the
start, dH, the accept decision and ok per trajectory, the CG bookkeeping and
the final sigma; the random stream is not stored: the GPU test draws it from
the same reference build, seeded the same way.

Only this script needs the reference tree; the fixture travels without it.
Usage: python tests/golden/make_chain.py
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle.oracle import Ref  # noqa: E402

L, SEED, BETA_S = 8, 1231, 0.85
CHAINS = {"readme": (0.2, 2, 1000), "reject": (1.0, 2, 500)}


def chain(name, eps, steps, ntraj):
    ref = Ref(L, 0)
    ref.init(SEED, BETA_S, eps, steps)
    sigma0 = np.random.default_rng(8).normal(0.0, np.sqrt(2.0 / (4 * BETA_S)), L ** 3)
    ref.set_sigma(sigma0)
    ref.lib.gnref_reset_counters()
    dH, acc, ok = np.zeros(ntraj), np.zeros(ntraj, np.int8), np.zeros(ntraj, np.int8)
    with tempfile.TemporaryDirectory() as td:
        accfile = str(Path(td) / "acc.txt")
        for t in range(ntraj):
            o, a, d = ref.trajectory(accfile)
            ok[t], acc[t], dH[t] = o, a, d
    print(name, "accepted", int(acc.sum()), "of", ntraj, "max |dH|", float(np.abs(dH).max()))
    return {f"{name}_{k}": v for k, v in dict(eps=eps, steps=steps, sigma0=sigma0, dH=dH, accepted=acc, ok=ok,
                                              counters=np.array(ref.counters()), sigma_final=ref.sigma()).items()}


def main():
    d = dict(L=L, seed=SEED, beta_s=BETA_S)
    for name, (eps, steps, ntraj) in CHAINS.items():
        d.update(chain(name, eps, steps, ntraj))
    np.savez_compressed(HERE / f"golden_L{L}_chains.npz", **d)


if __name__ == "__main__":
    main()
