"""Faults injected on the host, and the state the library leaves behind.

The reference's failure path: a CG that reaches its cap returns false
(conjugategradient.c:106), and the integrator restores sigma and its mass
before it returns false (moleculardynamics.c:1279-1284, and LeapFrog2Pi for
pi).  Here the cap is forced (an absolute tolerance of 1e-300 that no residual
reaches within V + 1 iterations) or a NaN is put into sigma; each test checks
the status, that the fields are back bit for bit, and that the context works
afterwards.  Serving admission is checked under a memory budget that holds
one request's work arrays at a time: requests queue instead of failing, a
request larger than the budget is refused with GN_ERR_ARG, and the results
equal those of a server with room to spare.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = 4
V = L ** 3
BETA = 0.85


def _fields(seed):
    rng = np.random.default_rng(seed)
    s = np.sqrt(2.0 / (4 * BETA))
    return rng, rng.normal(0, s, V), rng.normal(0, s, V)


def _gauss(rng, n=3 * V):
    """A draw function over n fresh N(0, 1) values (P, chi_0, chi_1)."""
    it = iter(rng.normal(size=n))
    return lambda: next(it)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_forced_cap_restores_sigma(port, precision):
    import gn_b200 as G
    prec = G.GN_PREC_FP64 if precision == "fp64" else G.GN_PREC_MIXED
    rng, sigma, _ = _fields(1)
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma)
        s0, sm0 = lat.store_sigma()
        r = lat.trajectory(BETA, 0.1, 3, _gauss(rng), None, tol_medium=1e-300, tol_high=1e-300, precision=prec)
        assert r["ok"] == 0
        s1, sm1 = lat.store_sigma()
        assert np.array_equal(s1, s0) and np.array_equal(sm1, sm0)
        assert np.array_equal(sm1, port.sigma_mass(L, s1))
        # the context runs a good trajectory next
        r = lat.trajectory(BETA, 0.1, 3, _gauss(rng), None, precision=prec)
        assert r["ok"] == 1


def test_forced_cap_restores_sigma_and_pi_u1():
    import gn_b200 as G
    rng, sigma, pi = _fields(2)
    draws = rng.normal(size=3 * V)
    pairs = rng.normal(size=(V // 2, 2))
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma)
        lat.load_pi(pi)
        s0, sm0 = lat.store_sigma()
        p0, pm0 = lat.store_pi()
        it = iter(draws)
        r = lat.trajectory(BETA, 0.1, 3, lambda: next(it), None, tol_medium=1e-300, tol_high=1e-300)
        assert r["ok"] == 0
        assert all(np.array_equal(a, b) for a, b in zip(lat.store_sigma(), (s0, sm0)))
        pit = iter(pairs)

        def pair(a, b):
            a[0], b[0] = next(pit)
        it = iter(draws)
        r = lat.trajectory_pi(BETA, 0.1, 3, pair, lambda: next(it), None, tol_high=1e-300)
        assert r["ok"] == 0
        assert all(np.array_equal(a, b) for a, b in zip(lat.store_pi(), (p0, pm0)))
        assert all(np.array_equal(a, b) for a, b in zip(lat.store_sigma(), (s0, sm0)))
        pit = iter(rng.normal(size=(V // 2, 2)))
        r = lat.trajectory_pi(BETA, 0.1, 3, pair, _gauss(rng, 2 * V), None)
        assert r["ok"] == 1


def test_nan_in_sigma():
    """A NaN in sigma: the first solve cannot converge and stops at its cap,
    the trajectory reports it (ok = 0) and leaves sigma as it was loaded, and
    the context runs normally once a finite sigma is loaded."""
    import gn_b200 as G
    rng, sigma, _ = _fields(3)
    bad = sigma.copy()
    bad[17] = np.nan
    with G.Lattice(L) as lat:
        lat.load_sigma(bad)
        r = lat.trajectory(BETA, 0.1, 3, _gauss(rng), None)
        assert r["ok"] == 0
        s1, _ = lat.store_sigma()
        assert np.isnan(s1[17]) and np.array_equal(np.delete(s1, 17), np.delete(bad, 17))
        sm = lat.sigma_mass(bad)
        x, info, st = lat.cg(sm, rng.normal(size=V), None, 1e-9, variant=1)
        assert st == G.GN_NOT_CONVERGED and info[0]["status"] != 1
        lat.load_sigma(sigma)
        r = lat.trajectory(BETA, 0.1, 3, _gauss(rng), None)
        assert r["ok"] == 1 and np.isfinite(r["dH"])


def test_serving_admission_under_a_small_budget():
    import gn_b200 as G
    params = G.Ensemble.params(0.08, 8)
    rng = np.random.default_rng(9)
    sig = [rng.normal(0, np.sqrt(2.0 / (4 * BETA)), 8 ** 3) for _ in range(2)]
    big = rng.normal(0, np.sqrt(2.0 / (4 * BETA)), 16 ** 3)
    out = {}
    for budget in (150_000, 8e9):  # 150 kB: one L = 8 request's work arrays (~100 kB), not two
        with G.Server(params, mem_budget_bytes=budget, seed=5) as s:
            cs = [s.add_chain(8, BETA, sig[c], stream_id=10 + c) for c in range(2)]
            c16 = s.add_chain(16, BETA, big, stream_id=30)
            ids = [s.submit(c, G.GN_REQ_TRAJECTORY) for c in cs]
            if budget < 1e6:
                with pytest.raises(G.GnError) as e:  # ~0.8 MB of work arrays: never admissible
                    s.submit(c16, G.GN_REQ_TRAJECTORY)
                assert e.value.status == G.GN_ERR_ARG
            peak = 0
            for _ in range(10000):
                s.step()
                ld = s.load()
                peak = max(peak, ld["running"])
                assert ld["bytes_in_use"] <= budget
                if ld["running"] == 0 and ld["queued"] == 0:
                    break
            info = [s.request(i) for i in ids]
            assert all(x["status"] == 2 and x["failed"] == 0 for x in info)
            if budget < 1e6:  # one at a time: the second is admitted once the first has retired
                assert peak == 1 and info[1]["t_admit"] >= info[0]["t_done"]
            out[budget] = ([x["dH"] for x in info], [s.chain_sigma(c) for c in cs])
    (dh_small, sg_small), (dh_big, sg_big) = out[150_000], out[8e9]
    assert dh_small == dh_big
    assert all(np.array_equal(a, b) for a, b in zip(sg_small, sg_big))
