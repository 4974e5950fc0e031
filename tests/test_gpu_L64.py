"""GPU parity at the benchmark's lattice size, L = 64 (V = 262,144), against
the reference's own code compiled at that size (oracle/_ref, built from the
reference's sources by oracle/build_ref.py), on the same host-generated fields
and with the reference's own dSFMT stream replayed.

What is compared, and to what bar:
  - sigma mass (sigma.c:75), M (dirac.c:46), out - M psi (dirac.c:213): bit-exact;
    M^T (dirac.c:88): 1e-15 relative (a gather instead of the scatter), and
    bit-exact in the exact-order mode;
  - the two-flavour CG on M M^T (conjugategradient.c:115 and :13) at the
    reference's absolute tolerance 1e-9: bit-identical solutions and
    iteration counts in GN_PREC_FP64_EXACT.  The fast FP64 path sums its
    global reductions as trees instead of the reference's serial loops, and
    CG carries that rounding forward: at this size the recursively updated
    residual of iteration ~340 differs enough that a solve may cross the
    absolute threshold one iteration earlier or later.  So there: iteration
    counts within one per solve and x to 1e-9 relative;
  - the sigma force (moleculardynamics.c:590-647): F, X and Y to 1e-9 (fast),
    bit-identical (exact), same counters;
  - the early-exit variant from a perturbed start at the loose tolerance 1e-3:
    the fast path stops within one iteration of the reference and both
    solutions meet the tolerance; they differ by ~1e-5 relative, a fraction
    of their own distance from the exact solution at that tolerance, so x is
    compared to 1e-4 there (bit for bit in exact mode);
  - one LFMN2VF trajectory, 10 x eps 0.05 (moleculardynamics.c:1234), with the
    reference's Gauss1 / Casuale as the draws.  With the reference's own
    tolerances (1e-3 for the MD forces, 1e-9 absolute at the ends), exact mode
    gives the same iteration count, dH as the reference prints it (%.16f) and
    sigma bit for bit.  The MD forces at 1e-3 carry solution differences of
    ~1e-5 (the item above) into dH at ~1e-4, so the fast FP64 and mixed paths
    are compared on the benchmark's workload instead: every solve to
    1e-10 |phi| (the reference built with GN_REF_RELATIVE_TOL, oracle/_ref
    libgnref_L64_i0_rel.so).  There they take the same accept decision, the
    same CG call count, iteration counts within one per solve, sigma to 1e-9
    and dH to 1e-7: at L = 64 the Hamiltonian is ~5e5, and the reference's
    own serial sum of V terms carries ~sqrt(V) * ulp(H) / 2 ~ 1e-8 of
    rounding in each of H0 and H1, while the GPU's compensated sums carry
    almost none.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = 64
V = L ** 3
BETA = 0.85
EXACT = 2
RTOL_FAST = 1e-9


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def ref():
    from oracle import build_ref
    from oracle.oracle import Ref
    if not build_ref.lib_path(L).exists() and not build_ref.available():
        pytest.skip("reference build oracle/_ref/libgnref_L64_i0.so not present")
    r = Ref(L)
    r.init(1231, BETA, 0.05, 10)
    return r


@pytest.fixture(scope="module")
def lat():
    import gn_b200 as G
    with G.Lattice(L) as lt:
        yield lt


@pytest.fixture(scope="module")
def fields(ref):
    """sigma ~ N(0, 2/(N_f beta_s)) on the dual sites and phi_f = M chi_f with
    chi ~ N(0, 1) real, formed by the reference itself."""
    rng = np.random.default_rng(64)
    sigma = rng.normal(0.0, np.sqrt(2.0 / (4 * BETA)), V)
    ref.set_sigma(sigma)
    sm = ref.sigmamass()
    chi = rng.normal(size=(2, V))
    phi = np.stack([ref.dirac(chi[f].astype(complex), 0).real for f in range(2)])
    return dict(sigma=sigma, sm=sm, chi=chi, phi=phi, psi=rng.normal(size=V), out0=rng.normal(size=V))


def test_L64_operators(ref, lat, fields):
    import gn_b200 as G
    sm = lat.sigma_mass(fields["sigma"])
    assert np.array_equal(sm, fields["sm"])
    psi = fields["psi"]
    assert np.array_equal(lat.dirac(sm, psi, G.GN_OP_M), ref.dirac(psi.astype(complex), 0).real)
    mt_ref = ref.dirac(psi.astype(complex), 1).real
    assert rel(lat.dirac(sm, psi, G.GN_OP_MT), mt_ref) <= 1e-15
    sub_ref = ref.dirac(psi.astype(complex), 2, out=fields["out0"].astype(complex)).real
    assert np.array_equal(lat.dirac(sm, psi, G.GN_OP_SUB_M, out=fields["out0"]), sub_ref)
    lat.set_parity_mode(True)
    try:
        assert np.array_equal(lat.dirac(sm, psi, G.GN_OP_MT), mt_ref)
    finally:
        lat.set_parity_mode(False)


def test_L64_cg_two_flavours(ref, lat, fields, port):
    sm, phi = fields["sm"], fields["phi"]
    xr, its = [], []
    for f in range(2):
        it0, _ = ref.counters()
        x, ok = ref.cg(phi[f].astype(complex), None, 1e-9, 1, f)
        assert ok
        xr.append(x.real)
        its.append(ref.counters()[0] - it0)
    x, info, st = lat.cg(sm, phi, None, 1e-9, variant=1)
    assert st == 0
    for f in range(2):
        assert abs(info[f]["iterations"] - its[f]) <= 1
        assert rel(x[f], xr[f]) < RTOL_FAST
    xe, infoe, st = lat.cg(sm, phi, None, 1e-9, variant=1, precision=EXACT)
    assert st == 0
    for f in range(2):
        assert infoe[f]["iterations"] == its[f]
        assert np.array_equal(xe[f], xr[f])
    # the early-exit variant from a perturbed start (conjugategradient.c:13), tolerance 1e-3
    rng = np.random.default_rng(5)
    x0 = xr[0] + 1e-3 * rng.normal(size=V)
    it0, _ = ref.counters()
    x3, ok = ref.cg(phi[0].astype(complex), x0.astype(complex), 1e-3, 0, 0)
    it3 = ref.counters()[0] - it0
    xg, info, st = lat.cg(sm, phi[0], x0, 1e-3, variant=0)
    assert st == 0 and abs(info[0]["iterations"] - it3) <= 1
    assert rel(xg, x3.real) < 1e-4
    r = phi[0] - port.dirac(L, sm, port.dirac(L, sm, xg, 1), 0)
    assert np.linalg.norm(r) < 1e-3
    xg, info, st = lat.cg(sm, phi[0], x0, 1e-3, variant=0, precision=EXACT)
    assert info[0]["iterations"] == it3 and np.array_equal(xg, x3.real)


def test_L64_mixed_true_residual(lat, fields, port):
    """The benchmark's solve: both flavours to a true relative residual of
    1e-10, FP64 and mixed, checked with the CPU restatement's operator."""
    import gn_b200 as G
    sm, phi = fields["sm"], fields["phi"]
    for prec in (G.GN_PREC_FP64, G.GN_PREC_MIXED):
        x, info, st = lat.cg(sm, phi, None, 1e-10, variant=1, relative=True, precision=prec)
        assert st == 0
        for f in range(2):
            r = phi[f] - port.dirac(L, sm, port.dirac(L, sm, x[f], 1), 0)
            assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(phi[f]) * 1.01


def test_L64_force(ref, lat, fields):
    sigma, sm, phi = fields["sigma"], fields["sm"], fields["phi"]
    ref.set_sigma(sigma)
    for f in range(2):
        ref.kit_set("phi", f, phi[f].astype(complex))
        ref.kit_set("X", f, np.zeros(V, complex))
    it0, c0 = ref.counters()
    assert ref.force(1e-9)
    it1, c1 = ref.counters()
    Fr = ref.force_buf()
    Xr = np.stack([ref.kit_get("X", f).real for f in range(2)])
    Yr = np.stack([ref.kit_get("Y", f).real for f in range(2)])
    F, X, Y, info, st = lat.sigma_force(BETA, sigma, sm, phi, np.zeros((2, V)), 1e-9)
    assert st == 0
    assert abs(sum(i["iterations"] for i in info) - (it1 - it0)) <= 2
    assert sum(i["counted"] for i in info) == c1 - c0
    assert rel(F, Fr) < RTOL_FAST and rel(X, Xr) < RTOL_FAST and rel(Y, Yr) < RTOL_FAST
    F, X, Y, info, st = lat.sigma_force(BETA, sigma, sm, phi, np.zeros((2, V)), 1e-9, precision=EXACT)
    assert st == 0
    assert np.array_equal(X, Xr) and np.array_equal(Y, Yr) and np.array_equal(F, Fr)


@pytest.fixture(scope="module")
def ref_rel():
    """The reference built with every CG stopped at 1e-10 |phi| (the benchmark's rule)."""
    from oracle import build_ref
    from oracle.oracle import Ref
    if not build_ref.lib_path(L, 0, build_ref.REL_TAG).exists() and not build_ref.available():
        pytest.skip("reference build oracle/_ref/libgnref_L64_i0_rel.so not present")
    r = Ref(L, 0, extra_defs=build_ref.REL_DEFS, tag=build_ref.REL_TAG, build=build_ref.available())
    r.init(1231, BETA, 0.05, 10)
    return r


def test_L64_trajectory_exact(ref, lat, fields, tmp_path):
    """One LFMN2VF trajectory, 10 x eps 0.05, from the same sigma, with the
    reference's tolerances: GN_PREC_FP64_EXACT drawing from the reference's
    own Gauss1 / Casuale after its dSFMT state is put back."""
    sigma0 = fields["sigma"]
    gauss, casuale = ref.fn_ptrs()
    ref.set_sigma(sigma0)
    ref.rng_save()
    it0, c0 = ref.counters()
    ok, acc, dH = ref.trajectory(str(tmp_path / "acc.txt"))
    it1, c1 = ref.counters()
    assert ok
    ref.rng_restore()
    lat.load_sigma(sigma0)
    r = lat.trajectory(BETA, 0.05, 10, gauss, casuale, precision=EXACT)
    assert r["ok"] == 1 and r["accepted"] == int(acc)
    assert (r["cg_iterations"], r["cg_calls"]) == (it1 - it0, c1 - c0)
    assert float(f"{r['dH']:.16f}") == dH
    assert np.array_equal(lat.store_sigma()[0], ref.sigma())


def test_L64_trajectory_benchmark_workload(ref_rel, lat, fields, tmp_path):
    """The benchmark's trajectory (every solve to 1e-10 |phi|): the fast FP64
    path and the mixed-precision path against the reference's own run."""
    import gn_b200 as G
    ref = ref_rel
    sigma0 = fields["sigma"]
    gauss, casuale = ref.fn_ptrs()
    ref.set_sigma(sigma0)
    ref.rng_save()
    it0, c0 = ref.counters()
    ok, acc, dH = ref.trajectory(str(tmp_path / "acc.txt"))
    it1, c1 = ref.counters()
    assert ok
    sig_ref = ref.sigma()
    for prec in (G.GN_PREC_FP64, G.GN_PREC_MIXED):
        ref.rng_restore()
        lat.load_sigma(sigma0)
        r = lat.trajectory(BETA, 0.05, 10, gauss, casuale, tol_medium=1e-10, tol_high=1e-10, relative=True,
                           precision=prec)
        sig = lat.store_sigma()[0]
        diag = (prec, r["cg_iterations"], it1 - it0, r["dH"], dH, rel(sig, sig_ref))
        assert r["ok"] == 1 and r["accepted"] == int(acc), diag
        assert r["cg_calls"] == c1 - c0, diag
        if prec == G.GN_PREC_FP64:
            assert abs(r["cg_iterations"] - (it1 - it0)) <= c1 - c0, diag
        assert abs(r["dH"] - dH) < 1e-7, diag
        assert rel(sig, sig_ref) < 1e-9, diag
