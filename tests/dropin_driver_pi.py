"""Runs the reference's PI_INTERACTION build with the U(1) drop-in library
interposed, in a fresh process; prints one JSON line.  Used by
tests/test_gpu_dropin.py.

libgn_dropin_pi.so is loaded first with RTLD_GLOBAL, then the reference's code
compiled with -DPI_INTERACTION (oracle/_ref/libgnref_L{L}_i0_pi.so).  The
harness then calls the reference's functions by name (DiracFermion, the CG,
ComputeSigmaForce, ComputePiForce, the energies, CondensateSigmaPi,
LeapFrog2MinimumNormSigmaVelocityFirst, LeapFrog2Pi, ComputeCondensateDirac) in the order
tests/golden/make_golden_u1.py called them on the reference alone, then
EvolveSigmaInTimeMinimumNormSigmaVelocityFirst on seeded inputs; each binds
to the drop-in's GPU version.  Random numbers come from the reference's own
Gauss1, Casuale and Gauss2MeanVariance, found by name.

usage: python tests/dropin_driver_pi.py <golden U(1) .npz> [exact]
("exact" selects GN_PREC_FP64_EXACT, the reference's order of operations)
"""
import ctypes as C
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def evolve_inputs_pi(L):
    """sigma, pi, P and chi of the MD-helper check (seeded)."""
    rng = np.random.default_rng(12)
    V = L ** 3
    w = np.sqrt(2.0 / (4 * 0.85))
    return rng.normal(0.0, w, V), rng.normal(0.0, w, V), rng.normal(size=V), rng.normal(size=(2, V))


def evolve_setup(ref, L, beta_s):
    """The reference's state for EvolveSigmaInTimeMinimumNormSigmaVelocityFirst:
    sigma, pi, P, phi_f = M chi_f and X_f = 0, counters reset."""
    sig0, pi0, P0, chi = evolve_inputs_pi(L)
    ref.init(1231, beta_s, 0.1, 4)
    ref.set_pi_params(0.1, 4)
    ref.set_sigma(sig0)
    ref.set_pi(pi0)
    ref.set_momenta(P0)
    for f in range(2):
        ref.kit_set("phi", f, ref.dirac(chi[f].astype(complex), 0))
        ref.kit_set("X", f, np.zeros(L ** 3, complex))
    ref.lib.gnref_reset_counters()


def main():
    g = dict(np.load(sys.argv[1]))
    L = int(g["L"])
    V = L ** 3
    drop = C.CDLL(str(ROOT / "3d-gross-neveu-model_b200" / "lib" / "libgn_dropin_pi.so"), mode=C.RTLD_GLOBAL)
    drop.GNB200_SetLattice(L)
    if len(sys.argv) > 2 and sys.argv[2] == "exact":
        drop.GNB200_SetPrecision(2)  # GN_PREC_FP64_EXACT
    drop.GNB200_Context.restype = C.c_void_p
    core = C.CDLL(str(ROOT / "3d-gross-neveu-model_b200" / "lib" / "libgn_b200.so"))
    core.gn_launch_count.restype = C.c_longlong
    core.gn_launch_count.argtypes = [C.c_void_p]
    launches = lambda: core.gn_launch_count(drop.GNB200_Context())  # noqa: E731  (GPU kernels so far)
    counts = {}
    from oracle import build_ref
    from oracle.oracle import Ref
    lib = C.CDLL(str(build_ref.lib_path(L, 0, build_ref.PI_TAG)), mode=C.RTLD_GLOBAL)
    ref = Ref(L, 0, build=False, extra_defs=build_ref.PI_DEFS, tag=build_ref.PI_TAG)
    ref.init(1231, float(g["beta_s"]), 0.1, 3)
    ref.set_pi_params(0.1, 3)
    ref.set_sigma(g["sigma"])
    ref.set_pi(g["pi"])
    out = {"pm": ref.pimass().tolist(), "sigma_obs": ref.condensate_sigma().tolist()}
    cj = lambda z: [np.real(z).tolist(), np.imag(z).tolist()]  # noqa: E731
    n0 = launches()
    out["M_psi"] = cj(ref.dirac(g["psi"], 0))
    counts["dirac"] = launches() - n0
    out["Mt_psi"] = cj(ref.dirac(g["psi"], 1))
    out["sub_res"] = cj(ref.dirac(g["psi"], 2, out=g["sub_out0"]))
    ref.lib.gnref_reset_counters()
    n0 = launches()
    x, ok = ref.cg(g["cg_b"], None, 1e-9, 1)
    counts["cg"] = launches() - n0
    out.update(cg_x=cj(x), cg_ok=bool(ok), cg_counters=list(ref.counters()))
    for f in range(2):
        ref.kit_set("phi", f, g["force_phi"][f])
        ref.kit_set("X", f, np.zeros(V, complex))
    ref.lib.gnref_reset_counters()
    out["force_ok"] = bool(ref.force(1e-9))
    out["force_F"] = ref.force_buf().tolist()
    out["force_X"] = [cj(ref.kit_get("X", f)) for f in range(2)]
    out["force_counters"] = list(ref.counters())
    for f in range(2):
        ref.kit_set("X", f, np.zeros(V, complex))
    n0 = launches()
    out["piforce_ok"] = bool(ref.pi_force())
    counts["pi_force"] = launches() - n0
    out["piforce_F"] = ref.pi_force_buf().tolist()
    out["piforce_Y"] = [cj(ref.kit_get("Y", f)) for f in range(2)]
    ref.set_momenta(g["energy_P"])
    ref.set_pi_momenta(g["energy_Ppi"])
    out["energy_H"] = ref.energy()
    out["energy_Hpi"] = ref.energy_pi()
    with tempfile.TemporaryDirectory() as td:
        accfile = str(Path(td) / "acc.txt")
        for name, run in (("traj", ref.trajectory), ("trajpi", ref.trajectory_pi)):
            ref.lib.gnref_reset_counters()
            n0 = launches()
            ok, accepted, dH = run(accfile)
            counts[name] = launches() - n0
            out.update({f"{name}_ok": bool(ok), f"{name}_dH": dH, f"{name}_accepted": int(accepted),
                        f"{name}_counters": list(ref.counters()), f"{name}_sigma": ref.sigma().tolist(),
                        f"{name}_pi": ref.pi().tolist()})
    # ComputeCondensateDirac on the state the trajectories left
    ref.kit_set("Y", 0, g["cond_target0"])
    ref.lib.gnref_reset_counters()
    n0 = launches()
    out["cond_out"] = ref.condensate(1e-9).tolist()
    counts["condensate"] = launches() - n0
    out.update(cond_counters=list(ref.counters()), cond_target=cj(ref.kit_get("Y", 0)),
               cond_D=cj(ref.kit_get("D", 0)))
    # the MD helper of the reference's reversibility check through its call site
    evolve_setup(ref, L, float(g["beta_s"]))
    n0 = launches()
    ref.evolve_in_time(0, 0.1, 4)
    counts["evolve"] = launches() - n0
    out.update(evolve_sigma=ref.sigma().tolist(), evolve_P=ref.momenta().tolist(),
               evolve_counters=list(ref.counters()))
    out["launches"] = counts
    C.CDLL(None).fflush(None)  # LeapFrog2Pi's printed lines go out before the JSON line
    print(json.dumps(out))
    _ = (drop, lib)


if __name__ == "__main__":
    main()
