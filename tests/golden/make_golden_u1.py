"""Generate the U(1)-model fixtures of tests/golden/ from the reference itself.

The reference compiled with PI_INTERACTION (oracle/build_ref.py with
extra_defs -DPI_INTERACTION, driven through oracle/ref_harness.c) runs its own
complex-mass Dirac operator, CG, sigma and pi forces and energies, one
LeapFrog2MinimumNormSigmaVelocityFirst trajectory, one LeapFrog2Pi
trajectory and then ComputeCondensateDirac on seeded sigma and pi fields; the random streams the trajectories
consumed (Gauss1, the Gauss2MeanVariance pairs of the pi momenta and Casuale,
all from dSFMT) are recorded so the fixtures replay them without the
reference's RNG.

Only this script needs the reference tree; the fixtures travel without it.
Usage: python tests/golden/make_golden_u1.py
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
PI_DEFS = ("-DPI_INTERACTION",)


def field(L, seed):
    return np.random.default_rng(seed).normal(0.0, np.sqrt(2.0 / (NFLAV * BETA_S)), L ** 3)


def cplx(rng, V):
    return rng.normal(size=V) + 1j * rng.normal(size=V)


def fixture(L):
    ref = Ref(L, 0, extra_defs=PI_DEFS, tag="_pi")
    ref.init(1231, BETA_S, 0.1, 3)
    ref.set_pi_params(0.1, 3)
    V = L ** 3
    rng = np.random.default_rng(500 + L)
    sigma, pi = field(L, 11 + L), field(L, 13 + L)
    ref.set_sigma(sigma)
    ref.set_pi(pi)
    d = dict(L=L, beta_s=BETA_S, sigma=sigma, pi=pi, sm=ref.sigmamass(), pm=ref.pimass(),
             sigma_obs=ref.condensate_sigma())  # CondensateSigmaPi of |(sigma, pi)|
    # operators on a complex field
    psi, out0 = cplx(rng, V), cplx(rng, V)
    d.update(psi=psi, M_psi=ref.dirac(psi, 0), Mt_psi=ref.dirac(psi, 1), sub_out0=out0,
             sub_res=ref.dirac(psi, 2, out=out0))
    # CG from zero at 1e-9 (variant 1), b = M chi with chi real
    b = ref.dirac(rng.normal(size=V).astype(complex), 0)
    ref.lib.gnref_reset_counters()
    x, ok = ref.cg(b, None, 1e-9, 1)
    d.update(cg_b=b, cg_x=x, cg_ok=ok, cg_counters=np.array(ref.counters()))
    # forces at phi_f = M chi_f from X = 0, tol 1e-9
    phi = np.stack([ref.dirac(rng.normal(size=V).astype(complex), 0) for _ in range(2)])
    for f in range(2):
        ref.kit_set("phi", f, phi[f])
        ref.kit_set("X", f, np.zeros(V, complex))
    ref.lib.gnref_reset_counters()
    oks = ref.force(1e-9)
    d.update(force_phi=phi, force_ok=oks, force_F=ref.force_buf(),
             force_X=np.stack([ref.kit_get("X", f) for f in range(2)]),
             force_Y=np.stack([ref.kit_get("Y", f) for f in range(2)]), force_counters=np.array(ref.counters()))
    for f in range(2):
        ref.kit_set("X", f, np.zeros(V, complex))
    okp = ref.pi_force()  # ComputePiForce inverts at HIGH_PRECISION_INVERSION (1e-9)
    d.update(piforce_ok=okp, piforce_F=ref.pi_force_buf(),
             piforce_X=np.stack([ref.kit_get("X", f) for f in range(2)]),
             piforce_Y=np.stack([ref.kit_get("Y", f) for f in range(2)]))
    # energies at (P, phi, X)
    P, Ppi = rng.normal(size=V), rng.normal(size=V)
    ref.set_momenta(P)
    ref.set_pi_momenta(Ppi)
    d.update(energy_P=P, energy_H=ref.energy(), energy_Ppi=Ppi, energy_Hpi=ref.energy_pi())
    # one sigma trajectory and one pi trajectory, with the streams they drew
    with tempfile.TemporaryDirectory() as td:
        accfile = str(Path(td) / "acc.txt")
        for name, run in (("traj", ref.trajectory), ("trajpi", ref.trajectory_pi)):
            ref.lib.gnref_reset_counters()
            s0, p0 = ref.sigma(), ref.pi()
            ref.lib.gnref_rng_save()
            ok, accepted, dh = run(accfile)
            assert ok
            ref.lib.gnref_rng_restore()
            if name == "trajpi":  # the pi momenta are Gauss2MeanVariance pairs, then chi from Gauss1
                d["trajpi_pairs"] = ref.gauss2(V // 2)
                draws = ref.gauss(2 * V)
            else:
                draws = ref.gauss(3 * V)
            d.update({f"{name}_sigma0": s0, f"{name}_pi0": p0, f"{name}_gauss": draws,
                      f"{name}_uniform": ref.uniform(1), f"{name}_dH": dh, f"{name}_accepted": accepted,
                      f"{name}_counters": np.array(ref.counters()), f"{name}_sigma": ref.sigma(),
                      f"{name}_pi": ref.pi()})
    d.update(traj_eps=0.1, traj_steps=3)
    # ComputeCondensateDirac with the complex M on the state the trajectories
    # left, from a seeded starting target, with the uniforms its Z2 vectors drew
    target0 = 0.1 * cplx(rng, V)
    ref.kit_set("Y", 0, target0)
    ref.lib.gnref_reset_counters()
    d.update(cond_sigma=ref.sigma(), cond_pi=ref.pi(), cond_sm=ref.sigmamass(), cond_target0=target0)
    ref.lib.gnref_rng_save()
    out = ref.condensate(1e-9)
    ref.lib.gnref_rng_restore()
    d.update(cond_uniform=ref.uniform(6 * V), cond_out=out, cond_target=ref.kit_get("Y", 0),
             cond_D=ref.kit_get("D", 0), cond_counters=np.array(ref.counters()))
    np.savez_compressed(HERE / f"golden_L{L}_u1.npz", **d)
    print(HERE / f"golden_L{L}_u1.npz", "dH", d["traj_dH"], d["trajpi_dH"])


def main():
    for L in (4, 8):
        fixture(L)


if __name__ == "__main__":
    main()
