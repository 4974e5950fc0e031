"""Generate oracle_L128_dH.json: dH of one LFMN2VF trajectory (10 x eps 0.05)
at L = 128 from the CPU restatement (oracle/gn_oracle.c, bit-identical to the
reference's serial code), for the L = 128 mixed-precision case of bench.py.

The inputs are those bench.py's l128_case forms for each beta_s: with
rng = numpy.random.default_rng(int(100 * beta_s)),
    sigma = rng.normal(0, sqrt(2 / (N_f beta_s)), V), then
    draws = rng.normal(size=3 V): the momenta P, then chi_0 and chi_1,
drawn by the trajectory in the reference's order (moleculardynamics.c:781,
fermion.c:337).  Every CG stops at |r| < 1e-10 |b| (the GPU's relative rule).
A trajectory takes about 15 minutes on one core; the three run in parallel.

Usage: python tests/golden/make_l128_dH.py
"""
from __future__ import annotations

import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
L, EPS, STEPS, TOL = 128, 0.05, 10, 1e-10
BETAS = (0.7, 0.85, 1.0)


def one(beta):
    sys.path.insert(0, str(ROOT))
    from oracle.oracle import Port
    port = Port()
    V = L ** 3
    rng = np.random.default_rng(int(beta * 100))
    sigma = rng.normal(0.0, np.sqrt(2.0 / (4 * beta)), V)
    draws = rng.normal(size=3 * V)
    gp, up = port.replay(draws, np.array([0.5]))
    st = dict(sigma=sigma.copy(), sm=port.sigma_mass(L, sigma), P=np.zeros(V), F=np.zeros(V),
              chi=np.zeros((2, V)), phi=np.zeros((2, V)), X=np.zeros((2, V)), Y=np.zeros((2, V)))
    t0 = time.time()
    ok, dH, acc, H0, H1 = port.trajectory(L, beta, EPS, STEPS, st, gp, up, tol_med=-TOL, tol_high=-TOL)
    return {"beta_s": beta, "ok": ok, "dH": dH, "H0": H0, "H1": H1, "cg_iterations": st["iterations"],
            "cg_calls": st["calls"], "seconds": round(time.time() - t0, 1)}


def main():
    with mp.get_context("spawn").Pool(len(BETAS)) as pool:
        rows = pool.map(one, BETAS)
    out = {"L": L, "eps": EPS, "steps": STEPS, "tol_relative": TOL, "integrator": "LFMN2VF",
           "source": "oracle/gn_oracle.c (CPU restatement, serial FP64)", "rows": rows}
    (HERE / "oracle_L128_dH.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
