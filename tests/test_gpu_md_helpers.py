"""The reference's MD helpers of its reversibility check -- EvolveSigmaInTimeLF2
(moleculardynamics.c:1460), EvolveSigmaInTimeMinimumNormLF2 (:1489) and
EvolveSigmaInTimeMinimumNormSigmaVelocityFirst (:1551) -- on the GPU through
gn_evolve_sigma_in_time, against the reference's own helpers (oracle/_ref, the
reference compiled at L = 8) from the same sigma, momenta, phi and start X.

Bar: the CG counters equal; sigma, sigmamass, P, F, X and Y within 1e-11
relative on the fast FP64 path (the solves' global sums are trees instead of
the reference's serial loops), bit for bit in GN_PREC_FP64_EXACT.  Flipping P
and running the helper again brings sigma back (the reference's use of them).
The same for the U(1) model against the reference's PI_INTERACTION build
(complex M, complex phi, X and Y; L = 4).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L, V = 8, 512
EXACT = 2


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def ref():
    from oracle import build_ref
    from oracle.oracle import Ref
    if not build_ref.lib_path(L).exists() and not build_ref.available():
        pytest.skip("reference build oracle/_ref/libgnref_L8_i0.so not present")
    r = Ref(L)
    r.init(1231, 0.85, 0.1, 4)
    return r


def _state(seed):
    rng = np.random.default_rng(seed)
    return dict(sigma=rng.normal(0.0, np.sqrt(2.0 / (4 * 0.85)), V), P=rng.normal(size=V),
                chi=rng.normal(size=(2, V)), X0=rng.normal(size=(2, V)) * 0.3)


@pytest.mark.parametrize("integrator", [0, 1, 2])
def test_evolve_in_time_vs_reference(ref, integrator):
    import gn_b200 as G
    s = _state(40 + integrator)
    eps, steps = 0.1, 4
    ref.set_sigma(s["sigma"])
    phi = np.stack([ref.dirac(s["chi"][f].astype(complex), 0).real for f in range(2)])
    ref.set_momenta(s["P"])
    for f in range(2):
        ref.kit_set("phi", f, phi[f].astype(complex))
        ref.kit_set("X", f, s["X0"][f].astype(complex))
    it0, c0 = ref.counters()
    ref.evolve_in_time(integrator, eps, steps)
    it1, c1 = ref.counters()
    want = dict(sigma=ref.sigma(), sm=ref.sigmamass(), P=ref.momenta(), F=ref.force_buf(),
                X=np.stack([ref.kit_get("X", f).real for f in range(2)]),
                Y=np.stack([ref.kit_get("Y", f).real for f in range(2)]))
    with G.Lattice(L) as lat:
        for prec in (G.GN_PREC_FP64, EXACT):
            lat.load_sigma(s["sigma"])
            lat.write_state(G.GN_F_P, s["P"])
            lat.write_state(G.GN_F_PHI, phi.reshape(-1))
            lat.write_state(G.GN_F_X, s["X0"].reshape(-1))
            r = lat.evolve_in_time(0.85, eps, steps, integrator=integrator, precision=prec)
            assert r["ok"] == 1
            assert (r["cg_iterations"], r["cg_calls"]) == (it1 - it0, c1 - c0)
            assert abs(r["distance"] - eps * steps) < 1e-12
            sig, sm = lat.store_sigma()
            got = dict(sigma=sig, sm=sm, P=lat.read_state(G.GN_F_P), F=lat.read_state(G.GN_F_F),
                       X=lat.read_state(G.GN_F_X).reshape(2, V), Y=lat.read_state(G.GN_F_Y).reshape(2, V))
            for k in want:
                if prec == EXACT:
                    assert np.array_equal(got[k], want[k]), k
                else:
                    assert rel(got[k], want[k]) < 1e-11, k


@pytest.mark.parametrize("integrator", [0, 1, 2])
def test_evolve_in_time_reversible(integrator):
    """Evolve, flip P, evolve again: sigma comes back (DEBUG_LF2_SIGMA)."""
    import gn_b200 as G
    s = _state(70 + integrator)
    with G.Lattice(L) as lat:
        sm = lat.sigma_mass(s["sigma"])
        phi = np.stack([lat.dirac(sm, s["chi"][f], G.GN_OP_M) for f in range(2)])
        lat.load_sigma(s["sigma"])
        lat.write_state(G.GN_F_P, s["P"])
        lat.write_state(G.GN_F_PHI, phi.reshape(-1))
        lat.write_state(G.GN_F_X, np.zeros(2 * V))
        kw = dict(integrator=integrator, tol_medium=1e-12, tol_high=1e-12)
        lat.evolve_in_time(0.85, 0.1, 4, **kw)
        lat.write_state(G.GN_F_P, -lat.read_state(G.GN_F_P))
        lat.evolve_in_time(0.85, 0.1, 4, **kw)
        assert rel(lat.store_sigma()[0], s["sigma"]) < 1e-9
        assert rel(-lat.read_state(G.GN_F_P), s["P"]) < 1e-9


LU = 4


@pytest.fixture(scope="module")
def ref_pi():
    from oracle import build_ref
    from oracle.oracle import Ref
    if not build_ref.lib_path(LU, 0, build_ref.PI_TAG).exists():
        pytest.skip("reference PI build oracle/_ref/libgnref_L4_i0_pi.so not present")
    r = Ref(LU, 0, build=False, extra_defs=build_ref.PI_DEFS, tag=build_ref.PI_TAG)
    r.init(1231, 0.85, 0.1, 4)
    r.set_pi_params(0.1, 4)
    return r


def _planes(z):
    """complex (2, V) -> the four planes of both flavours (flavour f: 2f real, 2f + 1 imaginary)"""
    return np.concatenate([z[0].real, z[0].imag, z[1].real, z[1].imag])


@pytest.mark.parametrize("integrator", [0, 1, 2])
def test_evolve_in_time_u1_vs_reference(ref_pi, integrator):
    import gn_b200 as G
    V = LU ** 3
    rng = np.random.default_rng(90 + integrator)
    w = np.sqrt(2.0 / (4 * 0.85))
    sigma, pi, P = rng.normal(0.0, w, V), rng.normal(0.0, w, V), rng.normal(size=V)
    chi = rng.normal(size=(2, V))
    X0 = (rng.normal(size=(2, V)) + 1j * rng.normal(size=(2, V))) * 0.3
    eps, steps = 0.1, 4
    ref_pi.set_sigma(sigma)
    ref_pi.set_pi(pi)
    phi = np.stack([ref_pi.dirac(chi[f].astype(complex), 0) for f in range(2)])
    ref_pi.set_momenta(P)
    for f in range(2):
        ref_pi.kit_set("phi", f, phi[f])
        ref_pi.kit_set("X", f, X0[f])
    it0, c0 = ref_pi.counters()
    ref_pi.evolve_in_time(integrator, eps, steps)
    it1, c1 = ref_pi.counters()
    want = dict(sigma=ref_pi.sigma(), sm=ref_pi.sigmamass(), P=ref_pi.momenta(), F=ref_pi.force_buf(),
                X=_planes(np.stack([ref_pi.kit_get("X", f) for f in range(2)])),
                Y=_planes(np.stack([ref_pi.kit_get("Y", f) for f in range(2)])))
    assert np.array_equal(ref_pi.pi(), pi)  # the helpers leave pi alone
    with G.Lattice(LU) as lat:
        for prec in (G.GN_PREC_FP64, EXACT):
            lat.load_sigma(sigma)
            lat.load_pi(pi)
            lat.write_state(G.GN_F_P, P)
            lat.write_state(G.GN_F_PHI_C, _planes(phi))
            lat.write_state(G.GN_F_X_C, _planes(X0))
            r = lat.evolve_in_time(0.85, eps, steps, integrator=integrator, precision=prec)
            assert r["ok"] == 1
            assert (r["cg_iterations"], r["cg_calls"]) == (it1 - it0, c1 - c0)
            sig, sm = lat.store_sigma()
            got = dict(sigma=sig, sm=sm, P=lat.read_state(G.GN_F_P), F=lat.read_state(G.GN_F_F),
                       X=lat.read_state(G.GN_F_X_C).reshape(-1), Y=lat.read_state(G.GN_F_Y_C).reshape(-1))
            for k in want:
                if prec == EXACT:
                    assert np.array_equal(got[k], want[k]), k
                else:
                    assert rel(got[k], want[k]) < 1e-11, k
            assert np.array_equal(lat.store_pi()[0], pi)
