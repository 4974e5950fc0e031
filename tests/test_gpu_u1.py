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
    accept decision, the final fields to 1e-11.
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
