"""GN_PREC_FP64_EXACT: the GPU path in the reference's exact order of
operations (serial sums, M^T in the scatter's order, no FMA) reproduces the
reference's own results bit for bit -- solutions, iteration counts, forces,
every trajectory's dH and sigma, the condensate (whose chi_p solve is complex:
|z| there is the host library's own hypot, restated in csrc/host_hypot.h)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXACT = 2


@pytest.mark.parametrize("L", [4, 8, 16])
def test_exact_ops_vs_golden(golden, L):
    import gn_b200 as G
    g = golden(f"golden_L{L}_ops.npz")
    with G.Lattice(L) as lat:
        lat.set_parity_mode(True)
        sm = g["sm"]
        assert np.array_equal(lat.dirac(sm, g["psi"], G.GN_OP_MT), g["Mt_psi"])
        x1, info, st = lat.cg(sm, g["cg_b"], None, 1e-9, variant=1, precision=EXACT)
        assert st == 0 and info[0]["iterations"] == g["cg_it1"] and np.array_equal(x1, g["cg_x1"])
        x3, info, st = lat.cg(sm, g["cg_b3"], g["cg_x1"], 1e-3, variant=0, precision=EXACT)
        assert info[0]["iterations"] == g["cg_it3"] and np.array_equal(x3, g["cg_x3"])
        F, X, Y, info, st = lat.sigma_force(0.85, g["sigma"], sm, g["force_phi"], np.zeros((2, L ** 3)), 1e-9,
                                            precision=EXACT)
        assert np.array_equal(X, g["force_X"]) and np.array_equal(Y, g["force_Y"]) and np.array_equal(F, g["force_F"])
        assert lat.energy(0.85, g["sigma"], g["energy_P"], g["force_phi"], g["force_X"]) == float(g["energy_H"])


@pytest.mark.parametrize("name", ["golden_L8_hmc_i0.npz", "golden_L8_hmc_i1.npz", "golden_L8_hmc_i2.npz",
                                  "golden_L4_hmc_i0.npz"])
def test_exact_trajectories_vs_golden(port, golden, name):
    import gn_b200 as G
    g = golden(name)
    L = int(g["L"])
    gp, up = port.replay(g["gauss"], g["uniform"])
    with G.Lattice(L) as lat:
        lat.load_sigma(g["sigma0"])
        for t in range(len(g["dH"])):
            r = lat.trajectory(float(g["beta_s"]), float(g["eps"]), int(g["steps"]), gp, up,
                               integrator=int(g["integrator"]), precision=EXACT)
            assert float(f"{r['dH']:.16f}") == g["dH"][t]
            assert r["accepted"] == int(g["accepted"][t])
            assert np.array_equal(lat.store_sigma()[0], g["sigma_final"][t])
        assert np.array_equal(lat.read_state(G.GN_F_P), g["P_final"])
        assert np.array_equal(lat.read_state(G.GN_F_X), g["X_final"])
        assert np.array_equal(lat.read_state(G.GN_F_Y), g["Y_final"])


@pytest.mark.parametrize("L", [4, 8])
def test_exact_condensate_vs_golden(port, golden, L):
    import gn_b200 as G
    g = golden(f"golden_L{L}_cond.npz")
    _, up = port.replay(np.zeros(0), g["uniform"])
    with G.Lattice(L) as lat:
        out, target, D, it, calls, st = lat.condensate(g["sm"], 1e-9, g["target0"].astype(complex), up,
                                                       precision=EXACT)
    assert (it, calls) == tuple(g["counters"])
    assert np.array_equal(out, g["out"])
    assert np.array_equal(target, g["target"]) and np.array_equal(D, g["D"])


def test_exact_long_chain_vs_port(port):
    """200 chained trajectories, GPU exact mode against the CPU restatement
    (itself bit-identical to the reference): identical to the last bit."""
    import gn_b200 as G
    L, V, n = 8, 512, 200
    rng = np.random.default_rng(2024)
    gauss = rng.normal(size=n * 3 * V)
    unif = rng.uniform(size=n)
    sigma0 = rng.normal(0, np.sqrt(2 / (4 * 0.85)), V)
    gp, up = port.replay(gauss, unif)
    st = dict(sigma=sigma0.copy(), sm=port.sigma_mass(L, sigma0), P=np.zeros(V), F=np.zeros(V),
              chi=np.zeros((2, V)), phi=np.zeros((2, V)), X=np.zeros((2, V)), Y=np.zeros((2, V)))
    ref = [port.trajectory(L, 0.85, 0.2, 2, st, gp, up)[1] for _ in range(n)]
    gp, up = port.replay(gauss, unif)
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma0)
        got = [lat.trajectory(0.85, 0.2, 2, gp, up, precision=EXACT)["dH"] for _ in range(n)]
        s, _ = lat.store_sigma()
    assert got == ref
    assert np.array_equal(s, st["sigma"])
