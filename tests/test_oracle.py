"""CPU tests of the oracle: the restatement (oracle/gn_oracle.c) against the
golden fixtures made from the reference, and, where the reference tree is
present, against the reference's own code run live.  Bit-exact throughout."""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import build_ref
from oracle.oracle import OP_F_HIGH, OP_F_MED, OP_P, OP_Q, OP_S_HIGH

have_ref = build_ref.available()


def state_for(L, sigma, port):
    V = L ** 3
    return dict(sigma=sigma.copy(), sm=port.sigma_mass(L, sigma), P=np.zeros(V), F=np.zeros(V),
                chi=np.zeros((2, V)), phi=np.zeros((2, V)), X=np.zeros((2, V)), Y=np.zeros((2, V)))


@pytest.mark.parametrize("L", [4, 8, 16])
def test_port_ops_match_golden(port, golden, L):
    g = golden(f"golden_L{L}_ops.npz")
    sm = port.sigma_mass(L, g["sigma"])
    assert np.array_equal(sm, g["sm"])
    assert np.array_equal(port.dirac(L, sm, g["psi"], 0), g["M_psi"])
    assert np.array_equal(port.dirac(L, sm, g["psi"], 1), g["Mt_psi"])
    assert np.array_equal(port.dirac(L, sm, g["psi"], 2, out=g["sub_out0"]), g["sub_res"])
    x1, ok1, it1, cnt1 = port.cg(L, sm, g["cg_b"], None, 1e-9, 1)
    assert ok1 and cnt1 and it1 == g["cg_it1"] and np.array_equal(x1, g["cg_x1"])
    x2, ok2, it2, cnt2 = port.cg(L, sm, g["cg_b"], x1, 1e-9, 0)
    assert ok2 and not cnt2 and np.array_equal(x2, x1)  # early exit keeps x (conjugategradient.c:22-27)
    x3, ok3, it3, cnt3 = port.cg(L, sm, g["cg_b3"], x1, 1e-3, 0)
    assert ok3 and it3 == g["cg_it3"] and np.array_equal(x3, g["cg_x3"])
    F, X, Y, okf, itf, callsf = port.force(L, 0.85, g["sigma"], sm, g["force_phi"], np.zeros((2, L ** 3)), 1e-9)
    assert okf and np.array_equal(F, g["force_F"]) and np.array_equal(X, g["force_X"])
    assert np.array_equal(Y, g["force_Y"]) and (itf, callsf) == tuple(g["force_counters"])
    H = port.energy(L, 0.85, g["sigma"], g["energy_P"], g["force_phi"], g["force_X"])
    assert H == g["energy_H"]
    s, sme = port.evolve_sigma(L, g["sigma"], g["energy_P"], float(g["evolve_eps"]))
    assert np.array_equal(s, g["evolve_sigma"]) and np.array_equal(sme, g["evolve_sm"])
    assert np.array_equal(port.evolve_momenta(L, g["energy_P"], g["force_F"], 0.07), g["evolve_P"])


@pytest.mark.parametrize("name", ["golden_L8_hmc_i0.npz", "golden_L8_hmc_i1.npz", "golden_L8_hmc_i2.npz",
                                  "golden_L4_hmc_i0.npz"])
def test_port_trajectories_match_golden(port, golden, name):
    g = golden(name)
    L = int(g["L"])
    V = L ** 3
    gp, up = port.replay(g["gauss"], g["uniform"])
    st = state_for(L, g["sigma0"], port)
    for t in range(len(g["dH"])):
        ok, dH, acc, h0, h1 = port.trajectory(L, float(g["beta_s"]), float(g["eps"]), int(g["steps"]), st, gp, up,
                                              integrator=int(g["integrator"]))
        assert ok
        # the reference prints dH with %.16f (moleculardynamics.c:1426)
        assert float(f"{dH:.16f}") == g["dH"][t]
        assert acc == bool(g["accepted"][t])
        assert np.array_equal(st["sigma"], g["sigma_final"][t])
        assert (st["iterations"], st["calls"]) == tuple(g["counters"][t])
    assert port.replay_pos() == (len(g["gauss"]), len(g["uniform"]))
    assert np.array_equal(st["P"], g["P_final"]) and np.array_equal(st["F"], g["F_final"])
    assert np.array_equal(st["X"], g["X_final"]) and np.array_equal(st["Y"], g["Y_final"])
    assert np.array_equal(st["phi"], g["phi_final"])


@pytest.mark.parametrize("L", [4, 8])
def test_port_condensate_matches_golden(port, golden, L):
    g = golden(f"golden_L{L}_cond.npz")
    _, up = port.replay(np.zeros(0), g["uniform"])
    out, target, D, ok, it, calls = port.condensate(L, g["sm"], 1e-9, g["target0"].astype(complex), up)
    assert np.array_equal(out, g["out"])
    assert np.array_equal(target, g["target"]) and np.array_equal(D, g["D"])
    assert (it, calls) == tuple(g["counters"])


def test_schedules_force_counts(port):
    # LFMN2VF: 2 steps + 1 forces, the last at high precision (moleculardynamics.c:1234-1368)
    for steps in (2, 3, 10):
        ops, coefs = port.schedule(0, 0.05, steps)
        assert (ops == OP_F_MED).sum() == 2 * steps and (ops == OP_F_HIGH).sum() == 1
        assert np.isclose(coefs[ops == OP_Q].sum(), 0.05 * steps)
        assert np.isclose(coefs[ops == OP_P].sum(), 0.05 * steps)
    ops, coefs = port.schedule(1, 0.1, 4)  # LF2: steps + 1 forces
    assert (ops == OP_F_MED).sum() == 4 and (ops == OP_F_HIGH).sum() == 1
    ops, coefs = port.schedule(2, 0.1, 4)  # LFMN2: 2 steps forces + a final X0 solve
    assert (ops == OP_F_MED).sum() == 8 and (ops == OP_S_HIGH).sum() == 1
    assert np.isclose(coefs[ops == OP_Q].sum(), 0.4)


# ----------------------------------------------------------------- live reference
@pytest.mark.skipif(not have_ref, reason="reference tree not present")
@pytest.mark.parametrize("L", [4, 6, 8, 12, 16])
def test_reference_tables_closed_form(L):
    """The O(V) table fill of the harness equals StartLattice's O(V^2) one (lattice.c:225)."""
    from oracle.oracle import Ref
    ref = Ref(L)
    ref.init(1231, 0.85, 0.2, 2)
    assert ref.check_tables() == 0


@pytest.mark.skipif(not have_ref, reason="reference tree not present")
def test_port_tables_match_reference():
    from oracle.oracle import Port, Ref
    import ctypes as C
    port = Port()
    for L in (4, 6, 8):
        ref = Ref(L)
        ref.init(1231, 0.85, 0.2, 2)
        V = L ** 3
        site = np.zeros(V, np.int32)
        fpp = np.zeros(3 * V, np.int32)
        fmm = np.zeros(3 * V, np.int32)
        epp = np.zeros(3 * V)
        emm = np.zeros(3 * V)
        ip = C.POINTER(C.c_int)
        dp = C.POINTER(C.c_double)
        ref.lib.gnref_tables(site.ctypes.data_as(ip), fpp.ctypes.data_as(ip), fmm.ctypes.data_as(ip),
                             epp.ctypes.data_as(dp), emm.ctypes.data_as(dp))
        pp, mm, ep, em = port.tables(L)
        assert np.array_equal(pp.reshape(-1), fpp) and np.array_equal(mm.reshape(-1), fmm)
        assert np.array_equal(ep.reshape(-1).astype(float), epp) and np.array_equal(em.reshape(-1).astype(float), emm)


@pytest.mark.skipif(not have_ref, reason="reference tree not present")
@pytest.mark.parametrize("L,integrator,eps,steps,ntraj", [(6, 0, 0.2, 2, 6), (12, 0, 0.05, 4, 2), (8, 0, 0.2, 2, 100),
                                                          (6, 1, 0.1, 3, 4), (6, 2, 0.1, 3, 4)])
def test_port_equals_reference_live(port, L, integrator, eps, steps, ntraj):
    """Port and reference share one dSFMT stream: every trajectory and the
    following condensate must agree bit for bit."""
    from oracle.oracle import Ref
    ref = Ref(L, integrator)
    ref.init(1231, 0.85, eps, steps)
    rng = np.random.default_rng(L)
    sigma = rng.normal(0, np.sqrt(2 / (4 * 0.85)), L ** 3)
    ref.set_sigma(sigma)
    st = state_for(L, sigma, port)
    g, u = ref.fn_ptrs()
    with tempfile.TemporaryDirectory() as td:
        acc = str(Path(td) / "acc")
        n_acc = 0
        for _ in range(ntraj):
            ref.lib.gnref_rng_save()
            okr, accr, dHr = ref.trajectory(acc)
            ref.lib.gnref_rng_restore()
            okp, dHp, accp, _, _ = port.trajectory(L, 0.85, eps, steps, st, g, u, integrator=integrator)
            assert okr == okp and accr == accp and float(f"{dHp:.16f}") == dHr
            assert np.array_equal(ref.sigma(), st["sigma"])
            assert ref.counters() == (st["iterations"], st["calls"])
            n_acc += accr
    assert np.array_equal(ref.momenta(), st["P"])
    ref.lib.gnref_rng_save()
    cr = ref.condensate(1e-9)
    ref.lib.gnref_rng_restore()
    cp, tgt, D, ok, _, _ = port.condensate(L, st["sm"], 1e-9, st["Y"][0].astype(complex), u)
    assert np.array_equal(cr, cp)
