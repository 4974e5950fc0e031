"""GPU parity of the single-lattice operators, called through the C-ABI.

Reference results come from the golden fixtures (made by the reference's own
code) and from the bit-exact CPU restatement (oracle/gn_oracle.c) on larger
seeded inputs.  Tolerances:
  - sigma mass, M, out - M psi, the sigma / momentum steps: bit-exact (the FP64
    kernels keep the reference's order of operations and do not contract FMAs);
  - M^T: the gather adds the same seven exact terms in another order than the
    reference's scatter: |diff| <= 4 ulp of the largest term (rel. 1e-15);
  - CG solutions, forces: identical iteration counts; the solutions differ
    only through the order of the global sums (tree instead of serial), which
    CG amplifies by roughly the condition number: relative 1e-12 at L <= 16,
    1e-10 at L = 24;
  - energies: relative 1e-13.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_SOLVE = 1e-12


@pytest.fixture(scope="module")
def lattices():
    import gn_b200
    cache = {}

    def get(L):
        if L not in cache:
            cache[L] = gn_b200.Lattice(L)
        return cache[L]
    yield get
    for lat in cache.values():
        lat.close()


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("L", [4, 8, 16])
def test_ops_vs_golden(lattices, golden, L):
    import gn_b200 as G
    g = golden(f"golden_L{L}_ops.npz")
    lat = lattices(L)
    sm = lat.sigma_mass(g["sigma"])
    assert np.array_equal(sm, g["sm"])
    assert np.array_equal(lat.dirac(sm, g["psi"], G.GN_OP_M), g["M_psi"])
    assert rel(lat.dirac(sm, g["psi"], G.GN_OP_MT), g["Mt_psi"]) <= 1e-15
    assert np.array_equal(lat.dirac(sm, g["psi"], G.GN_OP_SUB_M, out=g["sub_out0"]), g["sub_res"])
    s, sme = lat.evolve_sigma(g["sigma"], g["energy_P"], float(g["evolve_eps"]))
    assert np.array_equal(s, g["evolve_sigma"]) and np.array_equal(sme, g["evolve_sm"])
    assert np.array_equal(lat.evolve_momenta(g["energy_P"], g["force_F"], 0.07), g["evolve_P"])


@pytest.mark.parametrize("L", [4, 8, 16])
def test_cg_vs_golden(lattices, golden, L):
    g = golden(f"golden_L{L}_ops.npz")
    lat = lattices(L)
    sm = g["sm"]
    x1, info, st = lat.cg(sm, g["cg_b"], None, 1e-9, variant=1)
    assert st == 0 and info[0]["counted"] and info[0]["iterations"] == g["cg_it1"]
    assert rel(x1, g["cg_x1"]) < RTOL_SOLVE
    # early exit on a start vector that already solves the system (conjugategradient.c:16-27)
    x2, info, st = lat.cg(sm, g["cg_b"], g["cg_x1"], 1e-9, variant=0)
    assert st == 0 and info[0]["status"] == 2 and not info[0]["counted"] and np.array_equal(x2, g["cg_x1"])
    x3, info, st = lat.cg(sm, g["cg_b3"], g["cg_x1"], 1e-3, variant=0)
    assert st == 0 and info[0]["iterations"] == g["cg_it3"]
    assert rel(x3, g["cg_x3"]) < 1e-10


@pytest.mark.parametrize("L", [4, 8, 16])
def test_force_energy_vs_golden(lattices, golden, L):
    g = golden(f"golden_L{L}_ops.npz")
    lat = lattices(L)
    F, X, Y, info, st = lat.sigma_force(0.85, g["sigma"], g["sm"], g["force_phi"], np.zeros((2, L ** 3)), 1e-9)
    assert st == 0
    assert (sum(i["iterations"] for i in info), sum(i["counted"] for i in info)) == tuple(g["force_counters"])
    assert rel(X, g["force_X"]) < RTOL_SOLVE and rel(Y, g["force_Y"]) < RTOL_SOLVE
    assert rel(F, g["force_F"]) < RTOL_SOLVE
    H = lat.energy(0.85, g["sigma"], g["energy_P"], g["force_phi"], g["force_X"])
    assert abs(H - float(g["energy_H"])) <= 1e-13 * abs(float(g["energy_H"]))


@pytest.mark.parametrize("L", [6, 12, 32])
def test_ops_vs_port_random(lattices, port, L):
    import gn_b200 as G
    rng = np.random.default_rng(L)
    V = L ** 3
    lat = lattices(L)
    sigma = rng.normal(0, 0.77, V)
    sm = lat.sigma_mass(sigma)
    assert np.array_equal(sm, port.sigma_mass(L, sigma))
    psi = rng.normal(size=V)
    assert np.array_equal(lat.dirac(sm, psi, G.GN_OP_M), port.dirac(L, sm, psi, 0))
    assert rel(lat.dirac(sm, psi, G.GN_OP_MT), port.dirac(L, sm, psi, 1)) <= 1e-15
    # complex planes: the operator acts on each plane
    z = psi + 1j * rng.normal(size=V)
    assert np.array_equal(lat.dirac(sm, z, G.GN_OP_M), port.dirac(L, sm, z, 0))
    # M^T is the transpose of M: <u, M v> = <M^T u, v>
    u, v = rng.normal(size=V), rng.normal(size=V)
    lhs = u @ lat.dirac(sm, v, G.GN_OP_M)
    rhs = lat.dirac(sm, u, G.GN_OP_MT) @ v
    assert abs(lhs - rhs) < 1e-11 * np.sqrt(V)


@pytest.mark.parametrize("L", [6, 12, 24])
def test_cg_multi_rhs_vs_port(lattices, port, L):
    """Two flavours solved in one kernel equal two separate reference solves."""
    rng = np.random.default_rng(3 * L)
    V = L ** 3
    lat = lattices(L)
    sm = lat.sigma_mass(rng.normal(0, 0.77, V))
    b = np.stack([port.dirac(L, sm, rng.normal(size=V), 0) for _ in range(2)])
    x, info, st = lat.cg(sm, b, None, 1e-9, variant=1)
    assert st == 0
    for k in range(2):
        xr, ok, it, cnt = port.cg(L, sm, b[k], None, 1e-9, 1)
        assert info[k]["iterations"] == it
        assert rel(x[k], xr) < (RTOL_SOLVE if L <= 16 else 1e-10)


def test_cg_complex_joint_vs_port(lattices, port):
    """A complex right-hand side is one joint system (shared alpha, beta), as the
    reference's complex CG on a real operator."""
    L = 8
    rng = np.random.default_rng(9)
    V = L ** 3
    lat = lattices(L)
    sm = lat.sigma_mass(rng.normal(0, 0.77, V))
    b = rng.normal(size=V) + 1j * rng.normal(size=V)
    x, info, st = lat.cg(sm, b, None, 1e-9, variant=1)
    xr, ok, it, cnt = port.cg(L, sm, b, None, 1e-9, 1)
    assert st == 0 and info[0]["iterations"] == it
    assert rel(x, xr) < RTOL_SOLVE


def test_cg_relative_stop_and_cap(lattices, port):
    L = 16
    rng = np.random.default_rng(4)
    V = L ** 3
    lat = lattices(L)
    sm = lat.sigma_mass(rng.normal(0, 0.77, V))
    b = port.dirac(L, sm, rng.normal(size=V), 0)
    x, info, st = lat.cg(sm, b, None, 1e-10, variant=1, relative=True)
    assert st == 0
    r = b - port.dirac(L, sm, port.dirac(L, sm, x, 1), 0)
    assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(b) * 1.01
    # the iteration cap returns the reference's `false` (conjugategradient.c:106)
    x, info, st = lat.cg(sm, b, None, 1e-14, variant=1, max_iter=5)
    assert st == 1 and info[0]["status"] == 3 and info[0]["iterations"] == 5


def test_mixed_precision_solver(lattices, port):
    """FP32 inner iterations + FP64 reliable updates reach the FP64 stopping rule
    on the true residual."""
    import gn_b200 as G
    L = 16
    rng = np.random.default_rng(12)
    V = L ** 3
    lat = lattices(L)
    sm = lat.sigma_mass(rng.normal(0, 0.77, V))
    b = np.stack([port.dirac(L, sm, rng.normal(size=V), 0) for _ in range(2)])
    x64, i64, st = lat.cg(sm, b, None, 1e-10, variant=1, relative=True)
    xm, im, st2 = lat.cg(sm, b, None, 1e-10, variant=1, relative=True, precision=G.GN_PREC_MIXED)
    assert st == 0 and st2 == 0
    for k in range(2):
        r = b[k] - port.dirac(L, sm, port.dirac(L, sm, xm[k], 1), 0)
        assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(b[k]) * 1.01
        assert im[k]["reliable_updates"] >= 1
        assert rel(xm[k], x64[k]) < 1e-8


@pytest.mark.parametrize("L", [96, 128])
def test_mixed_precision_schemes(lattices, port, L):
    """Both inner iterations of the mixed solver: the split (Chronopoulos-Gear)
    one at L = 96, whose FP32 vectors fit the L2, and the two-phase one at
    L = 128.  Each reaches the FP64 stopping rule on the true residual within
    a few per cent of the FP64 solver's iteration count; the FP64 solution's
    true residual is checked with the CPU restatement's operator as well."""
    import gn_b200 as G
    rng = np.random.default_rng(L)
    V = L ** 3
    lat = lattices(L)
    sm = lat.sigma_mass(rng.normal(0, 0.77, V))
    b = np.stack([rng.normal(size=V) for _ in range(2)])
    x64, i64, st = lat.cg(sm, b, None, 1e-10, variant=1, relative=True)
    xm, im, st2 = lat.cg(sm, b, None, 1e-10, variant=1, relative=True, precision=G.GN_PREC_MIXED)
    assert st == 0 and st2 == 0
    for k in range(2):
        # both solvers' true residuals, with the CPU restatement's operator
        for x in (x64[k], xm[k]):
            r = b[k] - port.dirac(L, sm, port.dirac(L, sm, x, 1), 0)
            assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(b[k]) * 1.01
        assert im[k]["iterations"] <= 1.1 * i64[k]["iterations"] + 20
        assert rel(xm[k], x64[k]) < 1e-7


@pytest.mark.parametrize("L", [6, 10])
def test_odd_half_rows_force_trajectory_mixed(lattices, port, L):
    """L/2 odd: every sweep runs one site per item (no 128-bit vectors).  The
    force and one LFMN2VF trajectory against the CPU restatement on the same
    random stream, and the mixed solver's true residual."""
    import gn_b200 as G
    rng = np.random.default_rng(100 + L)
    V = L ** 3
    lat = lattices(L)
    sigma = rng.normal(0, np.sqrt(2 / (4 * 0.85)), V)
    sm = lat.sigma_mass(sigma)
    phi = np.stack([port.dirac(L, sm, rng.normal(size=V), 0) for _ in range(2)])
    F, X, Y, info, st = lat.sigma_force(0.85, sigma, sm, phi, np.zeros((2, V)), 1e-9)
    Fr, Xr, Yr, ok, it, calls = port.force(L, 0.85, sigma, sm, phi, np.zeros((2, V)), 1e-9)
    assert st == 0 and ok and sum(i["iterations"] for i in info) == it
    assert rel(F, Fr) < RTOL_SOLVE and rel(X, Xr) < RTOL_SOLVE
    # one trajectory, GPU and port on the same draws
    gauss = rng.normal(size=3 * V)
    gp, up = port.replay(gauss, np.array([0.5]))
    st_port = dict(sigma=sigma.copy(), sm=sm.copy(), P=np.zeros(V), F=np.zeros(V), chi=np.zeros((2, V)),
                   phi=np.zeros((2, V)), X=np.zeros((2, V)), Y=np.zeros((2, V)))
    okp, dHp, accp, _, _ = port.trajectory(L, 0.85, 0.1, 3, st_port, gp, up)
    gp, up = port.replay(gauss, np.array([0.5]))
    lat.load_sigma(sigma)
    r = lat.trajectory(0.85, 0.1, 3, gp, up)
    assert okp and r["ok"] == 1 and r["accepted"] == int(accp)
    assert abs(r["dH"] - dHp) < 1e-10
    assert rel(lat.store_sigma()[0], st_port["sigma"]) < 1e-11
    # mixed precision: FP32 items of one site
    b = rng.normal(size=(2, V))
    xm, im, st = lat.cg(sm, b, None, 1e-10, variant=1, relative=True, precision=G.GN_PREC_MIXED)
    assert st == 0
    for k in range(2):
        r2 = b[k] - port.dirac(L, sm, port.dirac(L, sm, xm[k], 1), 0)
        assert np.linalg.norm(r2) < 1e-10 * np.linalg.norm(b[k]) * 1.01


@pytest.mark.parametrize("L", [16, 64])
def test_two_teams_and_lock_step_agree(port, monkeypatch, L):
    """The mixed solver's two flavours as two teams of half blocks (the
    default) and in lock step on all threads (GN_MIXED_DUO=0, read when a
    context is created): each system is the same CG, only the grouping of the
    partial sums differs, so both meet the FP64 stopping rule on the true
    residual with iteration counts within two of each other."""
    import gn_b200 as G
    rng = np.random.default_rng(600 + L)
    V = L ** 3
    sm = port.sigma_mass(L, rng.normal(0, 0.77, V))
    b = np.stack([port.dirac(L, sm, rng.normal(size=V), 0) for _ in range(2)])
    out = {}
    for duo in ("1", "0"):
        monkeypatch.setenv("GN_MIXED_DUO", duo)
        with G.Lattice(L) as lat:
            out[duo] = lat.cg(sm, b, None, 1e-10, variant=1, relative=True, precision=G.GN_PREC_MIXED)
    for duo, (x, info, st) in out.items():
        assert st == 0, duo
        for k in range(2):
            r = b[k] - port.dirac(L, sm, port.dirac(L, sm, x[k], 1), 0)
            assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(b[k]) * 1.01, (duo, k)
    for k in range(2):
        assert abs(out["1"][1][k]["iterations"] - out["0"][1][k]["iterations"]) <= 2
        assert rel(out["1"][0][k], out["0"][0][k]) < 1e-8
