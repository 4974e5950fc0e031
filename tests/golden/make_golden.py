"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own functions (compiled in place from the reference tree
by oracle/build_ref.py, driven through oracle/ref_harness.c) on seeded inputs
and stores inputs and outputs as .npz files.  The random streams the reference
consumed (its Gauss1 / Casuale outputs, from dSFMT seeded with Initrand) are
recorded too, so the fixtures can replay them without the reference's RNG.

Only this script needs the reference tree; the fixtures travel without it.
Usage: python tests/golden/make_golden.py
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


def sigma_init(L, seed):
    """sigma i.i.d. N(0, 2/(N_f beta_s)) on the dual sites, as the benchmark configs ask."""
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), L ** 3)


def ops_fixture(L):
    ref = Ref(L)
    ref.init(1231, BETA_S, 0.2, 2)
    V = L ** 3
    rng = np.random.default_rng(100 + L)
    sigma = sigma_init(L, L)
    ref.set_sigma(sigma)
    sm = ref.sigmamass()
    psi = rng.normal(size=V)
    out0 = rng.normal(size=V)
    d = dict(L=L, sigma=sigma, sm=sm, psi=psi)
    d["M_psi"] = ref.dirac(psi.astype(complex), 0).real
    d["Mt_psi"] = ref.dirac(psi.astype(complex), 1).real
    d["sub_out0"] = out0
    d["sub_res"] = ref.dirac(psi.astype(complex), 2, out=out0.astype(complex)).real
    # CG: b = M chi, x0 = 0 (variant 1) at 1e-9; then variant 0 restarted from that x (early exit)
    chi = rng.normal(size=V)
    b = ref.dirac(chi.astype(complex), 0)
    ref.lib.gnref_reset_counters()
    x1, ok1 = ref.cg(b, None, 1e-9, 1)
    it1, c1 = ref.counters()
    x2, ok2 = ref.cg(b, x1, 1e-9, 0)
    it2, c2 = ref.counters()
    # variant 0 at 1e-3 from a stale start (the solution of another right-hand side)
    b3 = ref.dirac(rng.normal(size=V).astype(complex), 0)
    x3, ok3 = ref.cg(b3, x1, 1e-3, 0)
    it3, c3 = ref.counters()
    d.update(cg_b=b.real, cg_x1=x1.real, cg_ok1=ok1, cg_it1=it1, cg_b3=b3.real, cg_x3=x3.real, cg_ok3=ok3,
             cg_it3=it3 - it2, cg_calls=np.array([c1, c2, c3]), cg_x2_equal=np.array_equal(x1, x2))
    # force at (sigma, phi) from zero start X, tol 1e-9
    phi = np.stack([ref.dirac(rng.normal(size=V).astype(complex), 0).real for _ in range(2)])
    for f in range(2):
        ref.kit_set("phi", f, phi[f].astype(complex))
        ref.kit_set("X", f, np.zeros(V, complex))
    ref.lib.gnref_reset_counters()
    okf = ref.force(1e-9)
    d.update(force_phi=phi, force_ok=okf, force_F=ref.force_buf(),
             force_X=np.stack([ref.kit_get("X", f).real for f in range(2)]),
             force_Y=np.stack([ref.kit_get("Y", f).real for f in range(2)]),
             force_counters=np.array(ref.counters()))
    # energy at (P, phi, X)
    P = rng.normal(size=V)
    ref.set_momenta(P)
    d.update(energy_P=P, energy_H=ref.energy())
    # evolve: sigma += eps P with sigma-mass recompute; P += eps F
    ref.evolve_sigma(0.05)
    d.update(evolve_eps=0.05, evolve_sigma=ref.sigma(), evolve_sm=ref.sigmamass())
    ref.evolve_momenta(0.07)
    d.update(evolve_P=ref.momenta())
    np.savez_compressed(HERE / f"golden_L{L}_ops.npz", **d)


def hmc_fixture(L, integrator, ntraj, eps, steps, seed=1231):
    ref = Ref(L, integrator)
    ref.init(seed, BETA_S, eps, steps)
    V = L ** 3
    sigma0 = sigma_init(L, 7 + L)
    ref.set_sigma(sigma0)
    gauss, unif, dH, acc, counters, sig_final = [], [], [], [], [], []
    with tempfile.TemporaryDirectory() as td:
        accfile = str(Path(td) / "acc.txt")
        for t in range(ntraj):
            ref.lib.gnref_rng_save()
            ok, accepted, dh = ref.trajectory(accfile)
            assert ok
            ref.lib.gnref_rng_restore()
            gauss.append(ref.gauss(3 * V))
            unif.append(ref.uniform(1))
            dH.append(dh)
            acc.append(accepted)
            counters.append(ref.counters())
            sig_final.append(ref.sigma())
    np.savez_compressed(HERE / f"golden_L{L}_hmc_i{integrator}.npz", L=L, integrator=integrator, eps=eps,
                        steps=steps, beta_s=BETA_S, sigma0=sigma0, gauss=np.concatenate(gauss),
                        uniform=np.concatenate(unif), dH=np.array(dH), accepted=np.array(acc),
                        counters=np.array(counters), sigma_final=np.stack(sig_final),
                        P_final=ref.momenta(), F_final=ref.force_buf(),
                        X_final=np.stack([ref.kit_get("X", f).real for f in range(2)]),
                        Y_final=np.stack([ref.kit_get("Y", f).real for f in range(2)]),
                        phi_final=np.stack([ref.kit_get("phi", f).real for f in range(2)]))


def condensate_fixture(L, seed=1231):
    ref = Ref(L)
    ref.init(seed, BETA_S, 0.2, 2)
    V = L ** 3
    sigma = sigma_init(L, 11 + L)
    ref.set_sigma(sigma)
    rng = np.random.default_rng(5 + L)
    target0 = rng.normal(size=V) * 0.1
    ref.kit_set("Y", 0, target0.astype(complex))
    ref.lib.gnref_reset_counters()
    ref.lib.gnref_rng_save()
    out = ref.condensate(1e-9)
    ref.lib.gnref_rng_restore()
    uniform = ref.uniform(6 * V)
    np.savez_compressed(HERE / f"golden_L{L}_cond.npz", L=L, sigma=sigma, sm=ref.sigmamass(), target0=target0,
                        uniform=uniform, out=out, target=ref.kit_get("Y", 0), D=ref.kit_get("D", 0),
                        counters=np.array(ref.counters()))


def layout_fixture():
    """The reference's struct layouts (sizes and member offsets) for the drop-in ABI check."""
    import ctypes as C
    ref = Ref(8)
    out = (C.c_long * 64)()
    n = ref.lib.gnref_layout(out)
    np.save(HERE / "layout_reference.npy", np.array(out[:n], dtype=np.int64))


def main():
    layout_fixture()
    for L in (4, 8, 16):
        ops_fixture(L)
    hmc_fixture(8, 0, 20, 0.2, 2)       # the README command line: beta_s 0.85, eps 0.2, 2 steps, seed 1231
    hmc_fixture(8, 1, 5, 0.2, 2)
    hmc_fixture(8, 2, 5, 0.2, 2)
    hmc_fixture(4, 0, 10, 0.05, 10)
    for L in (4, 8):
        condensate_fixture(L)
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
