"""The reference-signature drop-in (include/gn_dropin.h) interposed under the
reference's own code: the reference's harness calls its integrator, its
condensate and its Dirac operator by name, and the dynamic linker binds them to
the GPU versions.  With the reference's own dSFMT stream (seed 1231) the
results must equal the golden fixtures made by the reference alone: dH to
1e-10, every accept/reject decision, sigma to 1e-12, the CG counters.

Runs in a subprocess so that no earlier test has bound the reference's
symbols in this process.  Needs the reference build under oracle/_ref/ (made
by __graft_entry__.build() where the reference tree exists)."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"


def evolve_reference(L, beta_s, integrator):
    """The reference's own EvolveSigmaInTime* (no drop-in in this process) on the
    driver's inputs: (sigma, P, counters)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from dropin_driver import evolve_inputs

    from oracle.oracle import Ref
    ref = Ref(L, build=False)
    sig0, P0, chi = evolve_inputs(L)
    ref.init(1231, beta_s, 0.1, 4)
    ref.set_sigma(sig0)
    ref.set_momenta(P0)
    for f in range(2):
        ref.kit_set("phi", f, ref.dirac(chi[f].astype(complex), 0))
        ref.kit_set("X", f, np.zeros(L ** 3, complex))
    ref.lib.gnref_reset_counters()
    ref.evolve_in_time(integrator, 0.1, 4)
    return ref.sigma(), ref.momenta(), list(ref.counters())


def test_dropin_under_reference_driver(port):
    from oracle import build_ref
    if not build_ref.lib_path(8, 0).exists():
        pytest.skip("reference build oracle/_ref/libgnref_L8_i0.so not present")
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "dropin_driver.py"), str(GOLD / "golden_L8_hmc_i0.npz"),
                        str(GOLD / "golden_L8_cond.npz")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    g = dict(np.load(GOLD / "golden_L8_hmc_i0.npz"))
    assert np.max(np.abs(np.array(out["dH"]) - g["dH"])) < 1e-10
    assert out["accepted"] == [int(a) for a in g["accepted"]]
    assert max(out["sigma_rel"]) < 1e-12
    assert [tuple(c) for c in out["counters"]] == [tuple(c) for c in g["counters"]]
    c = dict(np.load(GOLD / "golden_L8_cond.npz"))
    for k in range(11):
        assert abs(out["condensate"][k] - c["out"][k]) <= 1e-11 * max(abs(c["out"][k]), 1e-3)
    assert tuple(out["condensate_counters"]) == tuple(c["counters"])
    # the replacement took effect: each phase launched the library's kernels
    assert all(out["launches"][k] > 0 for k in ("trajectories", "condensate", "dirac", "evolve")), out["launches"]
    assert out["launches"]["trajectories"] >= 20 * 5  # 20 trajectories, each with solves, forces and steps
    # DiracFermion called by the reference's harness equals the reference's own M, bit for bit
    L = 8
    assert np.array_equal(np.array(out["M_psi"]), port.dirac(L, np.array(out["sm"]), np.array(out["psi"]), 0))
    # EvolveSigmaInTimeMinimumNormSigmaVelocityFirst called by the reference's harness
    s_ref, P_ref, cnt_ref = evolve_reference(L, float(g["beta_s"]), int(g["integrator"]))
    assert out["evolve_counters"] == cnt_ref
    assert np.max(np.abs(np.array(out["evolve_sigma"]) - s_ref)) < 1e-12 * np.max(np.abs(s_ref))
    assert np.max(np.abs(np.array(out["evolve_P"]) - P_ref)) < 1e-11 * np.max(np.abs(P_ref))


def test_dropin_exact_mode_is_bit_identical():
    """GNB200_SetPrecision(GN_PREC_FP64_EXACT): the reference's driver code on
    the GPU reproduces the reference's own run bit for bit."""
    from oracle import build_ref
    if not build_ref.lib_path(8, 0).exists():
        pytest.skip("reference build oracle/_ref/libgnref_L8_i0.so not present")
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "dropin_driver.py"), str(GOLD / "golden_L8_hmc_i0.npz"),
                        str(GOLD / "golden_L8_cond.npz"), "exact"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    g = dict(np.load(GOLD / "golden_L8_hmc_i0.npz"))
    assert out["dH"] == [float(v) for v in g["dH"]]
    assert all(out["sigma_equal"])
    assert [tuple(c) for c in out["counters"]] == [tuple(c) for c in g["counters"]]
    c = dict(np.load(GOLD / "golden_L8_cond.npz"))
    assert out["condensate"] == [float(v) for v in c["out"]]
    s_ref, P_ref, cnt_ref = evolve_reference(8, float(g["beta_s"]), int(g["integrator"]))
    assert out["evolve_counters"] == cnt_ref
    assert out["evolve_sigma"] == s_ref.tolist() and out["evolve_P"] == P_ref.tolist()


def evolve_reference_pi(L, beta_s):
    """The PI build's own EvolveSigmaInTimeMinimumNormSigmaVelocityFirst (no
    drop-in in this process) on the PI driver's inputs: (sigma, P, counters)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from dropin_driver_pi import evolve_setup

    from oracle import build_ref
    from oracle.oracle import Ref
    ref = Ref(L, 0, build=False, extra_defs=build_ref.PI_DEFS, tag=build_ref.PI_TAG)
    evolve_setup(ref, L, beta_s)
    ref.evolve_in_time(0, 0.1, 4)
    return ref.sigma(), ref.momenta(), list(ref.counters())


def _cx(a):
    return np.array(a[0]) + 1j * np.array(a[1])


def _run_pi_driver(L, *mode):
    from oracle import build_ref
    if not build_ref.lib_path(L, 0, build_ref.PI_TAG).exists():
        pytest.skip("reference PI build not present")
    gold = GOLD / f"golden_L{L}_u1.npz"
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "dropin_driver_pi.py"), str(gold), *mode],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    return json.loads(line), dict(np.load(gold))


@pytest.mark.parametrize("L", [4, 8])
def test_dropin_pi_exact_mode_is_bit_identical(L):
    """GNB200_SetPrecision(GN_PREC_FP64_EXACT) in libgn_dropin_pi.so: the
    reference's PI harness, calling its own functions by name, gets every
    result of its PI build bit for bit from the GPU."""
    out, g = _run_pi_driver(L, "exact")
    assert all(v > 0 for v in out["launches"].values()) and len(out["launches"]) == 7, out["launches"]
    for key in ("M_psi", "Mt_psi", "sub_res", "cg_x", "cond_target", "cond_D"):
        assert np.array_equal(_cx(out[key]), g[key]), key
    for key in ("force_X", "piforce_Y"):
        assert np.array_equal(np.stack([_cx(v) for v in out[key]]), g[key]), key
    for key in ("force_F", "piforce_F", "cond_out"):
        assert np.array_equal(np.array(out[key]), g[key]), key
    assert out["energy_H"] == g["energy_H"] and out["energy_Hpi"] == g["energy_Hpi"]
    assert tuple(out["cg_counters"]) == tuple(g["cg_counters"])
    assert tuple(out["cond_counters"]) == tuple(g["cond_counters"])
    for name in ("traj", "trajpi"):
        assert out[f"{name}_ok"] and out[f"{name}_dH"] == float(g[f"{name}_dH"])
        assert out[f"{name}_accepted"] == int(g[f"{name}_accepted"])
        assert tuple(out[f"{name}_counters"]) == tuple(g[f"{name}_counters"])
        assert np.array_equal(np.array(out[f"{name}_sigma"]), g[f"{name}_sigma"])
        assert np.array_equal(np.array(out[f"{name}_pi"]), g[f"{name}_pi"])
    s_ref, P_ref, cnt_ref = evolve_reference_pi(L, float(g["beta_s"]))
    assert out["evolve_counters"] == cnt_ref
    assert np.array_equal(np.array(out["evolve_sigma"]), s_ref) and np.array_equal(np.array(out["evolve_P"]), P_ref)


@pytest.mark.parametrize("L", [4, 8])
def test_dropin_pi_under_reference_harness(L):
    """libgn_dropin_pi.so under the reference's PI_INTERACTION build: the
    reference's harness calls its own U(1) functions by name and gets the
    GPU's, with the reference's RNG.  Results against the fixtures the
    reference made alone, to the tolerances of tests/test_gpu_u1.py."""
    out, g = _run_pi_driver(L)
    cx = _cx

    def rel(a, b):
        return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
    # the replacement took effect: each call site launched the library's kernels
    assert all(v > 0 for v in out["launches"].values()) and len(out["launches"]) == 7, out["launches"]
    assert np.array_equal(np.array(out["pm"]), g["pm"])
    np.testing.assert_allclose(out["sigma_obs"], g["sigma_obs"], rtol=1e-12, atol=1e-16)
    assert np.array_equal(cx(out["M_psi"]), g["M_psi"])
    assert rel(cx(out["Mt_psi"]), g["Mt_psi"]) < 1e-15
    assert np.array_equal(cx(out["sub_res"]), g["sub_res"])
    assert out["cg_ok"] and tuple(out["cg_counters"]) == tuple(g["cg_counters"])
    assert rel(cx(out["cg_x"]), g["cg_x"]) < 1e-11
    assert out["force_ok"] and tuple(out["force_counters"]) == tuple(g["force_counters"])
    assert rel(np.array(out["force_F"]), g["force_F"]) < 1e-11
    assert rel(np.stack([cx(v) for v in out["force_X"]]), g["force_X"]) < 1e-11
    assert out["piforce_ok"]
    assert rel(np.array(out["piforce_F"]), g["piforce_F"]) < 1e-11
    assert rel(np.stack([cx(v) for v in out["piforce_Y"]]), g["piforce_Y"]) < 1e-11
    assert abs(out["energy_H"] - g["energy_H"]) < 1e-13 * abs(g["energy_H"])
    assert abs(out["energy_Hpi"] - g["energy_Hpi"]) < 1e-13 * abs(g["energy_Hpi"])
    for name in ("traj", "trajpi"):
        assert out[f"{name}_ok"]
        assert abs(out[f"{name}_dH"] - float(g[f"{name}_dH"])) < 1e-10
        assert out[f"{name}_accepted"] == int(g[f"{name}_accepted"])
        assert tuple(out[f"{name}_counters"]) == tuple(g[f"{name}_counters"])
        assert rel(np.array(out[f"{name}_sigma"]), g[f"{name}_sigma"]) < 1e-11
        assert rel(np.array(out[f"{name}_pi"]), g[f"{name}_pi"]) < 1e-11
    # the condensate with the complex M
    assert tuple(out["cond_counters"]) == tuple(g["cond_counters"])
    for k in range(11):
        assert abs(out["cond_out"][k] - g["cond_out"][k]) <= 1e-11 * max(abs(g["cond_out"][k]), 1e-3), k
    assert rel(cx(out["cond_target"]), g["cond_target"]) < 1e-11
    assert rel(cx(out["cond_D"]), g["cond_D"]) < 1e-11
    # the MD helper through its call site
    s_ref, P_ref, cnt_ref = evolve_reference_pi(L, float(g["beta_s"]))
    assert out["evolve_counters"] == cnt_ref
    assert rel(np.array(out["evolve_sigma"]), s_ref) < 1e-11 and rel(np.array(out["evolve_P"]), P_ref) < 1e-11
