"""Failure detection on the GPU without a GPU fault.

A wait on other blocks that never ends (a block or peer that died) must end
with an error status the host reads, leaving the context usable; and a host
thread must be able to stop a running solve.  Both are made to happen here by
ordinary means: the library's own bounded team barrier run for a team whose
second block is never launched (gn_selftest_wait_timeout), and an abort
request from a second host thread during a solve that cannot converge (a
tolerance of 0).  Nothing traps, faults or spins without a bound: the barrier
gives up after its poll limit (about a second), and the solve would end at
its iteration cap (a few seconds) if the abort were not seen.
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_context_survives(port):
    import gn_b200 as G
    L = 8
    rng = np.random.default_rng(5)
    with G.Lattice(L) as lat:
        t0 = time.perf_counter()
        st = lat.selftest_wait_timeout()
        dt = time.perf_counter() - t0
        assert st == G.GN_ERR_TIMEOUT and dt < 30.0
        # the same context solves as before
        sm = lat.sigma_mass(rng.normal(0.0, 0.77, L ** 3))
        b = rng.normal(size=L ** 3)
        x, info, st = lat.cg(sm, b, None, 1e-9, variant=1)
        xr, ok, it, _ = port.cg(L, sm, b, None, 1e-9, 1)
        assert st == G.GN_OK and info[0]["iterations"] == it
        assert np.max(np.abs(x - xr)) <= 1e-12 * np.max(np.abs(xr))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_abort_stops_a_running_solve(precision):
    import gn_b200 as G
    prec = G.GN_PREC_FP64 if precision == "fp64" else G.GN_PREC_MIXED
    L = 32
    rng = np.random.default_rng(6)
    with G.Lattice(L) as lat:
        sm = lat.sigma_mass(rng.normal(0.0, 0.77, L ** 3))
        b = rng.normal(size=(2, L ** 3))
        out = {}

        def solve():
            t0 = time.perf_counter()
            try:  # tolerance 0: runs until the abort (or the cap of 300,000 iterations)
                _, _, st = lat.cg(sm, b, None, 0.0, variant=1, max_iter=300_000, precision=prec)
                out["status"] = st
            except G.GnError as e:
                out["status"] = e.status
            out["s"] = time.perf_counter() - t0
        th = threading.Thread(target=solve)
        th.start()
        time.sleep(0.5)
        lat.request_abort(True)
        th.join(timeout=120)
        assert not th.is_alive()
        lat.request_abort(False)
        assert out["status"] == G.GN_ERR_ABORTED, out
        # the context solves again once the request is withdrawn
        x, info, st = lat.cg(sm, b, None, 1e-10, variant=1, relative=True, precision=prec)
        assert st == G.GN_OK and all(i["status"] == 1 for i in info)
