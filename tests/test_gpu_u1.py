"""GPU parity of the U(1) Gross-Neveu model (the reference's PI_INTERACTION)
against fixtures made by the reference compiled with PI_INTERACTION
(tests/golden/make_golden_u1.py), through the C-ABI.

Tolerances, as for the Z2 model (tests/test_gpu_ops.py):
  - pi mass, M and out - M psi with the complex mass: bit-exact (FP64 without
    FMA contraction, the complex products formed as C forms them);
  - M^dagger: the gather adds the reference's scatter terms in another order:
    relative 1e-15;
  - CG solutions and forces: identical iteration counts, relative 1e-11 (the
    global sums run in a tree, which CG amplifies);
  - energies: relative 1e-13; trajectories: dH to 1e-10 absolute, the same
    accept decision, the final fields to 1e-11;
  - in the exact-order mode (GN_PREC_FP64_EXACT) every one of these bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("L", [4, 8])
def test_u1_operators_solve_forces_energies(golden, L):
    import gn_b200 as G
    g = golden(f"golden_L{L}_u1.npz")
    beta = float(g["beta_s"])
    with G.Lattice(L) as lat:
        lat.load_sigma(g["sigma"])
        lat.load_pi(g["pi"])
        _, pm = lat.store_pi()
        assert np.array_equal(pm, g["pm"])
        # CondensateSigmaPi of the U(1) order parameter |(sigma, pi)|
        np.testing.assert_allclose(lat.condensate_sigma(), g["sigma_obs"], rtol=1e-12, atol=1e-16)
        sm = g["sm"]
        assert np.array_equal(lat.dirac_u1(sm, pm, g["psi"], G.GN_OP_M), g["M_psi"])
        assert rel(lat.dirac_u1(sm, pm, g["psi"], G.GN_OP_MT), g["Mt_psi"]) < 1e-15
        assert np.array_equal(lat.dirac_u1(sm, pm, g["psi"], G.GN_OP_SUB_M, out=g["sub_out0"]), g["sub_res"])
        # CG from zero
        x, info, st = lat.cg_u1(sm, pm, g["cg_b"], None, 1e-9, variant=1)
        assert st == G.GN_OK and bool(g["cg_ok"])
        assert info[0]["iterations"] == g["cg_counters"][0]
        assert rel(x, g["cg_x"]) < 1e-11
        # forces from X = 0
        zero = np.zeros((2, L ** 3), complex)
        F, X, Y, infos, st = lat.sigma_force_u1(beta, g["sigma"], sm, pm, g["force_phi"], zero, 1e-9)
        assert st == G.GN_OK
        assert sum(i["iterations"] for i in infos if i["counted"]) == g["force_counters"][0]
        assert rel(X, g["force_X"]) < 1e-11 and rel(Y, g["force_Y"]) < 1e-11
        assert rel(F, g["force_F"]) < 1e-11
        F, X, Y, infos, st = lat.pi_force(beta, g["pi"], sm, pm, g["force_phi"], zero, 1e-9)
        assert st == G.GN_OK
        assert rel(X, g["piforce_X"]) < 1e-11 and rel(Y, g["piforce_Y"]) < 1e-11
        assert rel(F, g["piforce_F"]) < 1e-11
        # energies at the pi force's X
        H = lat.energy_u1(0, beta, g["sigma"], g["energy_P"], g["force_phi"], g["piforce_X"])
        assert abs(H - g["energy_H"]) < 1e-13 * abs(g["energy_H"])
        Hpi = lat.energy_u1(1, beta, g["pi"], g["energy_Ppi"], g["force_phi"], g["piforce_X"])
        assert abs(Hpi - g["energy_Hpi"]) < 1e-13 * abs(g["energy_Hpi"])


@pytest.mark.parametrize("L", [4, 8])
def test_u1_trajectories(golden, port, L):
    """One sigma trajectory (LFMN2VF with the complex M) and one LeapFrog2Pi,
    driven by the random streams the reference drew."""
    import gn_b200 as G
    g = golden(f"golden_L{L}_u1.npz")
    beta, eps, steps = float(g["beta_s"]), float(g["traj_eps"]), int(g["traj_steps"])
    with G.Lattice(L) as lat:
        lat.load_sigma(g["traj_sigma0"])
        lat.load_pi(g["traj_pi0"])
        gp, up = port.replay(g["traj_gauss"], g["traj_uniform"])
        r = lat.trajectory(beta, eps, steps, gp, up)
        assert r["ok"] == 1 and port.replay_pos() == (3 * L ** 3, 1)
        assert abs(r["dH"] - float(g["traj_dH"])) < 1e-10
        assert r["accepted"] == int(g["traj_accepted"])
        assert (r["cg_iterations"], r["cg_calls"]) == tuple(g["traj_counters"])
        assert rel(lat.store_sigma()[0], g["traj_sigma"]) < 1e-11
        lat.load_sigma(g["trajpi_sigma0"])
        lat.load_pi(g["trajpi_pi0"])
        gp, up = port.replay(g["trajpi_gauss"], g["trajpi_uniform"])
        pairs = iter(g["trajpi_pairs"])

        def pair(a, b):
            a[0], b[0] = next(pairs)
        r = lat.trajectory_pi(beta, eps, steps, pair, gp, up)
        assert r["ok"] == 1 and port.replay_pos() == (2 * L ** 3, 1)
        assert next(pairs, None) is None
        assert abs(r["dH"] - float(g["trajpi_dH"])) < 1e-10
        assert r["accepted"] == int(g["trajpi_accepted"])
        assert (r["cg_iterations"], r["cg_calls"]) == tuple(g["trajpi_counters"])
        assert rel(lat.store_pi()[0], g["trajpi_pi"]) < 1e-11
        assert np.array_equal(lat.store_sigma()[0], g["trajpi_sigma0"])  # LeapFrog2Pi leaves sigma alone


@pytest.mark.parametrize("L", [4, 8])
def test_u1_exact_order(golden, port, L):
    """GN_PREC_FP64_EXACT with the complex mass (M^dagger in the order of the
    reference's scatter, one-block solves with serial sums, serial energies):
    M^dagger, the solve, both forces, both energies, both trajectories and the
    condensate equal the reference's PI build bit for bit."""
    import gn_b200 as G
    g = golden(f"golden_L{L}_u1.npz")
    beta, eps, steps = float(g["beta_s"]), float(g["traj_eps"]), int(g["traj_steps"])
    EX = G.GN_PREC_FP64_EXACT
    with G.Lattice(L) as lat:
        lat.load_sigma(g["sigma"])
        lat.load_pi(g["pi"])
        sm, pm = g["sm"], g["pm"]
        lat.set_parity_mode(True)
        assert np.array_equal(lat.dirac_u1(sm, pm, g["psi"], G.GN_OP_MT), g["Mt_psi"])
        x, info, st = lat.cg_u1(sm, pm, g["cg_b"], None, 1e-9, variant=1, precision=EX)
        assert st == G.GN_OK and info[0]["iterations"] == g["cg_counters"][0]
        assert np.array_equal(x, g["cg_x"])
        zero = np.zeros((2, L ** 3), complex)
        F, X, Y, infos, st = lat.sigma_force_u1(beta, g["sigma"], sm, pm, g["force_phi"], zero, 1e-9)
        assert st == G.GN_OK
        assert sum(i["iterations"] for i in infos if i["counted"]) == g["force_counters"][0]
        assert np.array_equal(X, g["force_X"]) and np.array_equal(Y, g["force_Y"])
        assert np.array_equal(F, g["force_F"])
        F, X, Y, infos, st = lat.pi_force(beta, g["pi"], sm, pm, g["force_phi"], zero, 1e-9)
        assert st == G.GN_OK
        assert np.array_equal(X, g["piforce_X"]) and np.array_equal(Y, g["piforce_Y"])
        assert np.array_equal(F, g["piforce_F"])
        assert lat.energy_u1(0, beta, g["sigma"], g["energy_P"], g["force_phi"], g["piforce_X"]) == g["energy_H"]
        assert lat.energy_u1(1, beta, g["pi"], g["energy_Ppi"], g["force_phi"], g["piforce_X"]) == g["energy_Hpi"]
        lat.set_parity_mode(False)
        # the trajectories with the reference's draws
        lat.load_sigma(g["traj_sigma0"])
        lat.load_pi(g["traj_pi0"])
        gp, up = port.replay(g["traj_gauss"], g["traj_uniform"])
        r = lat.trajectory(beta, eps, steps, gp, up, precision=EX)
        # the fixture's dH is the reference's acceptance line, printed with %.16f
        assert r["ok"] == 1 and float(f"{r['dH']:.16f}") == float(g["traj_dH"])
        assert r["accepted"] == int(g["traj_accepted"])
        assert (r["cg_iterations"], r["cg_calls"]) == tuple(g["traj_counters"])
        assert np.array_equal(lat.store_sigma()[0], g["traj_sigma"])
        lat.load_sigma(g["trajpi_sigma0"])
        lat.load_pi(g["trajpi_pi0"])
        gp, up = port.replay(g["trajpi_gauss"], g["trajpi_uniform"])
        pairs = iter(g["trajpi_pairs"])

        def pair(a, b):
            a[0], b[0] = next(pairs)
        r = lat.trajectory_pi(beta, eps, steps, pair, gp, up, precision=EX)
        assert r["ok"] == 1 and float(f"{r['dH']:.16f}") == float(g["trajpi_dH"])
        assert r["accepted"] == int(g["trajpi_accepted"])
        assert (r["cg_iterations"], r["cg_calls"]) == tuple(g["trajpi_counters"])
        assert np.array_equal(lat.store_pi()[0], g["trajpi_pi"])
        # the condensate's ten solves and M^dagger applies
        _, up = port.replay(np.zeros(0), g["cond_uniform"])
        lat.load_sigma(g["cond_sigma"])
        lat.load_pi(g["cond_pi"])
        out, target, D, it, calls, st = lat.condensate(g["cond_sm"], 1e-9, g["cond_target0"], up, precision=EX)
    assert st == G.GN_OK and (it, calls) == tuple(g["cond_counters"])
    assert np.array_equal(out, g["cond_out"])
    assert np.array_equal(target, g["cond_target"]) and np.array_equal(D, g["cond_D"])


def test_u1_switch_back(golden):
    """gn_set_u1(0) returns the context to the Z2 model's real fields."""
    import gn_b200 as G
    g = golden("golden_L4_hmc_i0.npz")
    with G.Lattice(4) as lat:
        lat.load_pi(np.zeros(64))
        lat.set_u1(False)
        lat.load_sigma(g["sigma0"])
        r = lat.trajectory(float(g["beta_s"]), float(g["eps"]), int(g["steps"]), None, None)
        assert r["ok"] == 1


def _u1_fields(L, seed):
    rng = np.random.default_rng(seed)
    s = np.sqrt(2.0 / (4 * 0.85))
    return rng, rng.normal(0, s, L ** 3), rng.normal(0, s, L ** 3)


@pytest.mark.parametrize("L", [6, 16])
def test_u1_mixed_precision_solver(L):
    """The mixed solver with the complex mass (FP32 inner iterations, FP64
    reliable updates) meets the FP64 stopping rule on the true residual,
    checked with the FP64 operators, for one and two systems and both start
    variants."""
    import gn_b200 as G
    rng, sigma, pi = _u1_fields(L, 40 + L)
    V = L ** 3
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma)
        lat.load_pi(pi)
        _, pm = lat.store_pi()
        _, sm = lat.store_sigma()
        b = np.stack([rng.normal(size=V) + 1j * rng.normal(size=V) for _ in range(2)])
        x0 = 0.1 * (rng.normal(size=(2, V)) + 1j * rng.normal(size=(2, V)))
        for variant in (0, 1):
            for nsys in (1, 2):
                nb = b[0] if nsys == 1 else b
                start = None if variant == 1 else (x0[0] if nsys == 1 else x0)
                x64, i64, st = lat.cg_u1(sm, pm, nb, start, 1e-10, variant=variant, relative=True)
                xm, im, st2 = lat.cg_u1(sm, pm, nb, start, 1e-10, variant=variant, relative=True,
                                        precision=G.GN_PREC_MIXED)
                assert st == G.GN_OK and st2 == G.GN_OK
                bs, xs = np.atleast_2d(nb), np.atleast_2d(xm)
                for k in range(bs.shape[0]):
                    y = lat.dirac_u1(sm, pm, xs[k], G.GN_OP_MT)
                    r = bs[k] - lat.dirac_u1(sm, pm, y, G.GN_OP_M)
                    assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(bs[k]) * 1.01
                    assert im[k]["reliable_updates"] >= 1
                    assert im[k]["iterations"] <= 1.1 * i64[k]["iterations"] + 20
                assert rel(np.asarray(xm), np.asarray(x64)) < 1e-7


def test_u1_mixed_precision_trajectories(port):
    """Mixed-precision solves inside the U(1) sigma and pi trajectories: dH and
    the evolved fields agree with the FP64 path to the solver tolerance."""
    import gn_b200 as G
    L = 16
    V = L ** 3
    rng, sigma0, pi0 = _u1_fields(L, 91)
    gauss = rng.normal(size=3 * V)
    pairs = rng.normal(size=(V // 2, 2))
    unif = np.array([0.5])
    res = {}
    for prec in (G.GN_PREC_FP64, G.GN_PREC_MIXED):
        with G.Lattice(L) as lat:
            lat.load_sigma(sigma0)
            lat.load_pi(pi0)
            gp, up = port.replay(gauss, unif)
            r = lat.trajectory(0.85, 0.05, 4, gp, up, tol_medium=1e-10, tol_high=1e-10, relative=True,
                               precision=prec)
            it = iter(pairs)

            def pair(a, b):
                a[0], b[0] = next(it)
            gp, up = port.replay(gauss, unif)
            rp = lat.trajectory_pi(0.85, 0.05, 4, pair, gp, up, tol_high=1e-10, relative=True, precision=prec)
            res[prec] = (r, rp, lat.store_sigma()[0], lat.store_pi()[0])
    a, b = res[G.GN_PREC_FP64], res[G.GN_PREC_MIXED]
    for q in (0, 1):
        assert a[q]["ok"] and b[q]["ok"]
        assert abs(a[q]["dH"] - b[q]["dH"]) < 1e-6
        assert a[q]["accepted"] == b[q]["accepted"]
        assert b[q]["reliable_updates"] > 0
    assert rel(b[2], a[2]) < 1e-8 and rel(b[3], a[3]) < 1e-8


@pytest.mark.parametrize("L", [4, 8])
def test_u1_condensate(golden, port, L):
    """ComputeCondensateDirac of the reference's PI build (the same ten solves
    and M^dagger applies with the complex M), against its fixture: the 11
    outputs to 1e-11 relative, the reference's CG bookkeeping, and the final
    target and D to 1e-11."""
    import gn_b200 as G
    g = golden(f"golden_L{L}_u1.npz")
    _, up = port.replay(np.zeros(0), g["cond_uniform"])
    with G.Lattice(L) as lat:
        lat.load_sigma(g["cond_sigma"])
        lat.load_pi(g["cond_pi"])
        out, target, D, it, calls, st = lat.condensate(g["cond_sm"], 1e-9, g["cond_target0"], up)
    assert st == G.GN_OK
    assert port.replay_pos()[1] == 6 * L ** 3
    assert (it, calls) == tuple(g["cond_counters"])
    for k in range(11):
        assert abs(out[k] - g["cond_out"][k]) <= 1e-11 * max(abs(g["cond_out"][k]), 1e-3), (k, out[k])
    assert rel(target, g["cond_target"]) < 1e-11
    assert rel(D, g["cond_D"]) < 1e-11
