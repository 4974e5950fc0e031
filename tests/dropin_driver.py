"""Runs the reference's own driver functions with the drop-in library
interposed, in a fresh process; prints one JSON line.  Used by
tests/test_gpu_dropin.py.

The drop-in library (libgn_dropin.so) is loaded first with RTLD_GLOBAL, then
the reference's code (its sources compiled with -fPIC into
oracle/_ref/libgnref_L{L}_i0.so).  The reference's calls to its hot-path
functions (from its integrator, its harness entry points, its condensate)
go through the dynamic linker and bind to the drop-in's versions, which run on
the GPU; the random numbers come from the reference's own Gauss1 / Casuale,
found by name.

usage: python tests/dropin_driver.py <golden hmc .npz> <golden condensate .npz> [exact]
("exact" selects GN_PREC_FP64_EXACT, the reference's exact order of operations)
"""
import ctypes as C
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def evolve_inputs(L):
    """sigma, P and chi of the MD-helper check (seeded)."""
    rng = np.random.default_rng(11)
    V = L ** 3
    return rng.normal(0.0, np.sqrt(2.0 / (4 * 0.85)), V), rng.normal(size=V), rng.normal(size=(2, V))


def main():
    hmc = dict(np.load(sys.argv[1]))
    cond = dict(np.load(sys.argv[2]))
    L = int(hmc["L"])
    drop = C.CDLL(str(ROOT / "3d-gross-neveu-model_b200" / "lib" / "libgn_dropin.so"), mode=C.RTLD_GLOBAL)
    drop.GNB200_SetLattice(L)
    drop.GNB200_Context.restype = C.c_void_p
    core = C.CDLL(str(ROOT / "3d-gross-neveu-model_b200" / "lib" / "libgn_b200.so"))
    core.gn_launch_count.restype = C.c_longlong
    core.gn_launch_count.argtypes = [C.c_void_p]
    launches = lambda: core.gn_launch_count(drop.GNB200_Context())  # noqa: E731  (GPU kernels so far)
    if len(sys.argv) > 3 and sys.argv[3] == "exact":
        drop.GNB200_SetPrecision(2)
    from oracle import build_ref
    from oracle.oracle import Ref
    path = build_ref.lib_path(L, int(hmc["integrator"]))
    lib = C.CDLL(str(path), mode=C.RTLD_GLOBAL)  # the reference's code, with its Gauss1 / Casuale
    ref = Ref.__new__(Ref)
    Ref.__init__(ref, L, int(hmc["integrator"]), build=False)
    out = {"dH": [], "accepted": [], "sigma_rel": [], "counters": [], "launches": {}}
    ref.init(1231, float(hmc["beta_s"]), float(hmc["eps"]), int(hmc["steps"]))
    ref.set_sigma(hmc["sigma0"])
    n0 = launches()
    with tempfile.TemporaryDirectory() as td:
        acc = str(Path(td) / "acc.txt")
        for t in range(len(hmc["dH"])):
            ok, accepted, dH = ref.trajectory(acc)
            s = ref.sigma()
            out["dH"].append(dH)
            out.setdefault("sigma_equal", []).append(bool(np.array_equal(s, hmc["sigma_final"][t])))
            out["accepted"].append(int(accepted))
            out["sigma_rel"].append(float(np.max(np.abs(s - hmc["sigma_final"][t])) / np.max(np.abs(hmc["sigma_final"][t]))))
            out["counters"].append(list(ref.counters()))
    out["launches"]["trajectories"] = launches() - n0
    # the condensate through the reference's ComputeCondensateDirac call site
    ref.init(1231, float(hmc["beta_s"]), 0.2, 2)
    ref.set_sigma(cond["sigma"])
    ref.kit_set("Y", 0, cond["target0"].astype(complex))
    ref.lib.gnref_reset_counters()
    n0 = launches()
    out["condensate"] = ref.condensate(1e-9).tolist()
    out["launches"]["condensate"] = launches() - n0
    out["condensate_counters"] = list(ref.counters())
    # Dirac and CG through their call sites
    rng = np.random.default_rng(3)
    psi = rng.normal(size=L ** 3)
    n0 = launches()
    out["M_psi"] = ref.dirac(psi.astype(complex), 0).real.tolist()
    out["launches"]["dirac"] = launches() - n0
    out["psi"] = psi.tolist()
    out["sm"] = ref.sigmamass().tolist()
    # the MD helper of the reference's reversibility check (EvolveSigmaInTime*)
    # through its call site, on the inputs of evolve_inputs()
    sig0, P0, chi = evolve_inputs(L)
    ref.init(1231, float(hmc["beta_s"]), 0.1, 4)
    ref.set_sigma(sig0)
    ref.set_momenta(P0)
    for f in range(2):
        ref.kit_set("phi", f, ref.dirac(chi[f].astype(complex), 0))
        ref.kit_set("X", f, np.zeros(L ** 3, complex))
    ref.lib.gnref_reset_counters()
    n0 = launches()
    ref.evolve_in_time(int(hmc["integrator"]), 0.1, 4)
    out["launches"]["evolve"] = launches() - n0
    out["evolve_sigma"] = ref.sigma().tolist()
    out["evolve_P"] = ref.momenta().tolist()
    out["evolve_counters"] = list(ref.counters())
    print(json.dumps(out))
    _ = lib


if __name__ == "__main__":
    main()
