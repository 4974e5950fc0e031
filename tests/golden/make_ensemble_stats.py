"""Equilibrium statistics of the reference's own sigma-HMC chains, the
yardstick of the batched GPU chains (tests/test_gpu_ensemble.py).

For L (8 by default; 12 and 16 too) and beta_s in BETAS the reference
(compiled in place by oracle/build_ref.py, CG tolerances tightened to 1e-9
absolute, about 5e-11 relative at L = 8 and 1e-11 at L = 16) runs LFMN2VF
trajectories with eps = 0.08, 8 MD
steps, from sigma ~ N(0, 2/(N_f beta_s)), seed 1231: THERM trajectories of
thermalisation, then NMEAS measured ones.  Recorded per beta_s, each with an
error from binning:
  acceptance, <sigma^2> (site average after each trajectory), <exp(-dH)>,
  <|sigma_bar|> (|site average of sigma|), and the condensate tr1
  (ComputeCondensateDirac every COND_EVERY trajectories) oriented by the sign
  of sigma_bar: the model's Z2 symmetry maps sigma -> -sigma and tr1 -> -tr1,
  and a chain in the broken phase stays in one of the two vacua, so only the
  oriented value is comparable between chains.
The three beta_s run in parallel processes.
Output: tests/golden/ensemble_reference_L{L}.json.

Usage: python tests/golden/make_ensemble_stats.py [L]
"""
from __future__ import annotations

import json
import multiprocessing as mp
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle.oracle import Ref  # noqa: E402

L = int(sys.argv[1]) if len(sys.argv) > 1 and __name__ == "__main__" else 8
BETAS = (0.6, 0.85, 1.1)
EPS, STEPS = 0.08, 8
THERM, NMEAS, NBIN, COND_EVERY = 200, 2000, 20, 20
TIGHT = ("-DGN_REF_MEDIUM_TOL=1e-9", "-DGN_REF_HIGH_TOL=1e-9")


def binned(x, nbin=NBIN):
    x = np.asarray(x, float)
    b = x[: len(x) // nbin * nbin].reshape(nbin, -1).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(nbin))


def run(args):
    L, beta = args
    ref = Ref(L, 0, extra_defs=TIGHT, tag="_tight")
    ref.init(1231, beta, EPS, STEPS)
    rng = np.random.default_rng(int(beta * 1000))
    ref.set_sigma(rng.normal(0.0, np.sqrt(2.0 / (4 * beta)), L ** 3))
    acc, s2, emdh, sbar, cond = [], [], [], [], []
    with tempfile.TemporaryDirectory() as td:
        f = str(Path(td) / "acc.txt")
        for t in range(THERM + NMEAS):
            ok, a, dh = ref.trajectory(f)
            assert ok
            if t >= THERM:
                s = ref.sigma()
                acc.append(float(a))
                s2.append(float(np.mean(s ** 2)))
                sbar.append(float(abs(np.mean(s))))
                emdh.append(float(np.exp(-dh)))
                if (t - THERM) % COND_EVERY == COND_EVERY - 1:
                    cond.append(float(ref.condensate(1e-9)[0]) * float(np.sign(np.mean(s))))
    out = {"n": NMEAS}
    for name, x, nb in (("acceptance", acc, NBIN), ("sigma2", s2, NBIN), ("exp_mdH", emdh, NBIN),
                        ("abs_sigma_bar", sbar, NBIN), ("cond_tr1_oriented", cond, 10)):
        m, e = binned(x, nb)
        out[name] = m
        out[name + "_err"] = e
    return out


def main():
    res = {"L": L, "eps": EPS, "steps": STEPS, "integrator": 0, "therm": THERM, "betas": {}}
    Ref(L, 0, extra_defs=TIGHT, tag="_tight")  # build once, before the workers load it
    with mp.get_context("spawn").Pool(len(BETAS)) as pool:
        for b, r in zip(BETAS, pool.map(run, [(L, b) for b in BETAS])):
            res["betas"][str(b)] = r
            print(b, r, flush=True)
    (HERE / f"ensemble_reference_L{L}.json").write_text(json.dumps(res, indent=1) + "\n")


if __name__ == "__main__":
    main()
