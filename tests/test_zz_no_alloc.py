"""The allocation-free CG entry point (gn_cg_noalloc), called through the C-ABI.

Some callers cannot allocate device memory once they are running: an HMC
driver that sizes every buffer once up front, as the reference's Allocate*
functions do, or an application that gives the library a fixed budget from its
own pool allocator, where a cudaMalloc would escape the budget or fail.
gn_cg_noalloc keeps its scratch in a static device array instead of calling
cudaMalloc.  This test checks that two calls in a row give the same solution,
within the solver tolerance used by the other CG tests (relative 1e-12) and
with the same iteration counts, as the allocating entry point gn_cg_device --
from x = 0, from a start vector (the early-exit variant), with the relative
stopping rule -- that a call stopped by max_iter reports it and leaves nothing
behind for the next call, and that sizes beyond the static array's limit are
refused.  It creates its own contexts, so it passes alone in a fresh process as
well as after the other tests; its file name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_SOLVE = 1e-12


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def lib():
    import gn_b200
    lib = gn_b200.load_library()
    lib.gn_cg_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int,
                                  C.c_longlong, C.c_void_p, C.POINTER(gn_b200.CgInfo)]
    lib.gn_cg_noalloc.restype = C.c_int
    lib.gn_cg_noalloc_error.restype = C.c_char_p
    lib.gn_cg_noalloc_max_volume.restype = C.c_longlong
    return lib


@pytest.mark.parametrize("L", [8, 32])
def test_noalloc_matches_allocating_solver(lib, port, L):
    import gn_b200 as G
    V = L ** 3
    rng = np.random.default_rng(500 + L)
    sigma = rng.normal(0.0, np.sqrt(2.0 / (4 * 0.85)), V)
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma)
        sm = lat.field_ptr(G.GN_F_SM)
        # b in the first plane of PHI; the allocating solver writes X, the static-scratch one Y
        sm_h = port.sigma_mass(L, sigma)
        b = np.zeros((2, V))
        b[0] = port.dirac(L, sm_h, rng.normal(size=V), 0)
        lat.write_state(G.GN_F_PHI, b)
        lat.write_state(G.GN_F_X, np.zeros((2, V)))
        phi = lat.field_ptr(G.GN_F_PHI)
        infos_ref, st_ref = lat.cg_device(sm, phi, lat.field_ptr(G.GN_F_X), 1, 1, 1e-9, 1, False, 0,
                                          G.GN_PREC_FP64)
        assert st_ref == 0
        x_ref = lat.read_state(G.GN_F_X)[0]
        y = lat.field_ptr(G.GN_F_Y)
        for call in range(2):
            lat.write_state(G.GN_F_Y, np.full((2, V), 7.0))  # stale contents must not matter (x0 = 0)
            info = G.CgInfo()
            st = lib.gn_cg_noalloc(L, sm, phi, y, 1e-9, 1, 0, 0, lat.stream, C.byref(info))
            assert st == 0, lib.gn_cg_noalloc_error()
            x = lat.read_state(G.GN_F_Y)[0]
            assert info.iterations == infos_ref[0]["iterations"], call
            assert rel(x, x_ref) < RTOL_SOLVE, call
            # and it is a solution of the reference's system
            r = b[0] - port.dirac(L, sm_h, port.dirac(L, sm_h, x, 1), 0)
            assert np.linalg.norm(r) < 1e-9 * 1.01


def test_noalloc_rejects_oversize(lib):
    import gn_b200 as G
    assert lib.gn_cg_noalloc_max_volume() == 32 ** 3
    with G.Lattice(34) as lat:
        ptr = lat.field_ptr(G.GN_F_SM)
        st = lib.gn_cg_noalloc(34, ptr, lat.field_ptr(G.GN_F_PHI), lat.field_ptr(G.GN_F_X), 1e-9, 1, 0, 0,
                               lat.stream, None)
        assert st == -1
        assert b"static scratch limit" in lib.gn_cg_noalloc_error()


@pytest.mark.parametrize("variant,relative,tol", [(0, 0, 1e-9), (1, 1, 1e-10), (0, 1, 1e-10)])
def test_noalloc_start_vector_and_relative(lib, port, variant, relative, tol):
    """The early-exit variant from a non-zero start (conjugategradient.c:13)
    and the relative stopping rule, against gn_cg_device on the same input."""
    import gn_b200 as G
    L = 16
    V = L ** 3
    rng = np.random.default_rng(77 + variant + 2 * relative)
    sigma = rng.normal(0.0, np.sqrt(2.0 / (4 * 0.85)), V)
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma)
        sm = lat.field_ptr(G.GN_F_SM)
        sm_h = port.sigma_mass(L, sigma)
        b = np.zeros((2, V))
        b[0] = port.dirac(L, sm_h, rng.normal(size=V), 0)
        x0 = np.zeros((2, V))
        x0[0] = rng.normal(size=V) * 0.1
        lat.write_state(G.GN_F_PHI, b)
        lat.write_state(G.GN_F_X, x0)
        phi = lat.field_ptr(G.GN_F_PHI)
        infos_ref, st_ref = lat.cg_device(sm, phi, lat.field_ptr(G.GN_F_X), 1, 1, tol, variant, bool(relative), 0,
                                          G.GN_PREC_FP64)
        assert st_ref == 0
        x_ref = lat.read_state(G.GN_F_X)[0]
        y = lat.field_ptr(G.GN_F_Y)
        for call in range(2):
            lat.write_state(G.GN_F_Y, x0)
            info = G.CgInfo()
            st = lib.gn_cg_noalloc(L, sm, phi, y, tol, variant, relative, 0, lat.stream, C.byref(info))
            assert st == 0 and lib.gn_cg_noalloc_error() == b"", lib.gn_cg_noalloc_error()
            assert info.iterations == infos_ref[0]["iterations"], call
            assert rel(lat.read_state(G.GN_F_Y)[0], x_ref) < RTOL_SOLVE, call
        r = b[0] - port.dirac(L, sm_h, port.dirac(L, sm_h, lat.read_state(G.GN_F_Y)[0], 1), 0)
        bound = tol * (np.linalg.norm(b[0]) if relative else 1.0)
        assert np.linalg.norm(r) < bound * 1.01


def test_noalloc_iteration_cap_then_good_solve(lib, port):
    """max_iter stops a solve with GN_NOT_CONVERGED (the reference's `false`,
    conjugategradient.c:106); the next call starts clean and converges."""
    import gn_b200 as G
    L = 8
    V = L ** 3
    rng = np.random.default_rng(91)
    sigma = rng.normal(0.0, np.sqrt(2.0 / (4 * 0.85)), V)
    with G.Lattice(L) as lat:
        lat.load_sigma(sigma)
        sm = lat.field_ptr(G.GN_F_SM)
        sm_h = port.sigma_mass(L, sigma)
        b = np.zeros((2, V))
        b[0] = port.dirac(L, sm_h, rng.normal(size=V), 0)
        lat.write_state(G.GN_F_PHI, b)
        phi, y = lat.field_ptr(G.GN_F_PHI), lat.field_ptr(G.GN_F_Y)
        info = G.CgInfo()
        st = lib.gn_cg_noalloc(L, sm, phi, y, 1e-14, 1, 0, 5, lat.stream, C.byref(info))
        assert st == 1 and info.iterations == 5 and info.status == 3
        info = G.CgInfo()
        st = lib.gn_cg_noalloc(L, sm, phi, y, 1e-9, 1, 0, 0, lat.stream, C.byref(info))
        assert st == 0 and info.iterations > 5 and lib.gn_cg_noalloc_error() == b""
        xr, ok, it, _ = port.cg(L, sm_h, b[0], None, 1e-9, 1)
        assert ok and info.iterations == it
        assert rel(lat.read_state(G.GN_F_Y)[0], xr) < RTOL_SOLVE
