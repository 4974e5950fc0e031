"""Python front-end of the B200 fermion path (ctypes over include/gn_b200.h).

The product is the CUDA library lib/libgn_b200.so; this module only marshals
numpy arrays.  There is no CPU fallback: if the library cannot be loaded or no
sm_100 device is present, every call raises.

Fields are float64 arrays in the reference's fermion order (lexicographic
(x0*L + x1)*L + x2 with x2 = time fastest, even sites first).  Complex fields
(numpy complex128) are passed as two real planes.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libgn_b200.so"

GN_OK, GN_NOT_CONVERGED = 0, 1
GN_OP_M, GN_OP_MT, GN_OP_SUB_M = 0, 1, 2
GN_PREC_FP64, GN_PREC_MIXED, GN_PREC_FP64_EXACT = 0, 1, 2
GN_LFMN2VF, GN_LF2, GN_LFMN2 = 0, 1, 2
GN_F_P, GN_F_F, GN_F_CHI, GN_F_PHI, GN_F_X, GN_F_Y, GN_F_SIGMA, GN_F_SM = range(8)
# the U(1) model's resident fields: pi momenta and force (V), complex chi, phi,
# X, Y of both flavours (4V), and for field_ptr pi and pimass
GN_F_PI_P, GN_F_PI_F, GN_F_CHI_C, GN_F_PHI_C, GN_F_X_C, GN_F_Y_C, GN_F_PI, GN_F_PM = range(8, 16)
GN_ERR_ARG, GN_ERR_CUDA, GN_ERR_TIMEOUT, GN_ERR_ABORTED, GN_ERR_NO_DEVICE = -1, -2, -3, -4, -5
GN_ERR_IO, GN_ERR_NOT_FOUND, GN_ERR_FORMAT = -6, -7, -8
STATUS_NAMES = {0: "GN_OK", 1: "GN_NOT_CONVERGED", -1: "GN_ERR_ARG", -2: "GN_ERR_CUDA", -3: "GN_ERR_TIMEOUT",
                -4: "GN_ERR_ABORTED", -5: "GN_ERR_NO_DEVICE", -6: "GN_ERR_IO", -7: "GN_ERR_NOT_FOUND",
                -8: "GN_ERR_FORMAT"}
# CondensateSigmaPi's outputs (observables.c:323), in its argument order
SIGMA_OBSERVABLES = ("condensate_sigma", "condensate_sigma_abs", "mu2", "mu4", "chi", "chip", "chip_pbc1",
                     "chip_pbc2")
DRAW_FN = C.CFUNCTYPE(C.c_double)
PAIR_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double))


class GnError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class CgInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("counted", C.c_int), ("iterations", C.c_longlong), ("residual", C.c_double),
                ("b_norm", C.c_double), ("inner_iterations", C.c_longlong), ("reliable_updates", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class HmcParams(C.Structure):
    _fields_ = [("beta_s", C.c_double), ("eps", C.c_double), ("steps", C.c_int), ("integrator", C.c_int),
                ("tol_medium", C.c_double), ("tol_high", C.c_double), ("relative", C.c_int), ("precision", C.c_int)]


class TrajResult(C.Structure):
    _fields_ = [("ok", C.c_int), ("accepted", C.c_int), ("dH", C.c_double), ("H0", C.c_double), ("H1", C.c_double),
                ("cg_iterations", C.c_double), ("cg_calls", C.c_longlong), ("distance", C.c_double),
                ("inner_iterations", C.c_longlong), ("reliable_updates", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EnsParams(C.Structure):
    _fields_ = [("eps", C.c_double), ("steps", C.c_int), ("integrator", C.c_int), ("tol", C.c_double),
                ("precision", C.c_int)]


class ChainStats(C.Structure):
    _fields_ = [("trajectories", C.c_longlong), ("accepted", C.c_longlong), ("failed", C.c_longlong),
                ("cg_iterations", C.c_longlong), ("reliable_updates", C.c_longlong), ("sum_dH", C.c_double),
                ("sum_exp_mdH", C.c_double), ("sum_sigma2", C.c_double), ("last_dH", C.c_double),
                ("last_accepted", C.c_int), ("total_trajectories", C.c_longlong), ("total_accepted", C.c_longlong),
                ("story", C.c_int), ("local_accepted", C.c_int), ("local_done", C.c_int),
                ("epsilon_scale", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ReqInfo(C.Structure):
    _fields_ = [("id", C.c_longlong), ("type", C.c_int), ("status", C.c_int), ("chain", C.c_int),
                ("noise_vectors", C.c_int), ("failed", C.c_int), ("accepted", C.c_int), ("t_arrival", C.c_double),
                ("t_admit", C.c_double), ("t_done", C.c_double), ("dH", C.c_double), ("value", C.c_double),
                ("cg_iterations", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


GN_REQ_TRAJECTORY, GN_REQ_SOLVE, GN_REQ_CONDENSATE = 0, 1, 2


class HmcCounters(C.Structure):
    """The HMC bookkeeping of the reference's lattice file (gn_hmc_counters)."""
    _fields_ = [("epsilon_link", C.c_double), ("epsilon_pi", C.c_double), ("story_link", C.c_int),
                ("story_sigma", C.c_int), ("story_pi", C.c_int), ("accepted_link", C.c_int), ("done_link", C.c_int),
                ("accepted_sigma", C.c_int), ("done_sigma", C.c_int), ("accepted_pi", C.c_int),
                ("done_pi", C.c_int), ("measure", C.c_int)]

    @classmethod
    def from_dict(cls, d):
        return cls(**{k: (float if t is C.c_double else int)(d.get(k, 0)) for k, t in cls._fields_})

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_dp = C.POINTER(C.c_double)
_lib = None


def load_library(build_if_missing: bool = True) -> C.CDLL:
    """Load lib/libgn_b200.so (compiling it with nvcc first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists() and build_if_missing:
        import importlib.util
        spec = importlib.util.spec_from_file_location("gn_build", PKG / "build.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = C.CDLL(str(LIB_PATH))
    v = C.c_void_p
    sig = {
        "gn_create": ([C.POINTER(v), C.c_int, C.c_int], C.c_int),
        "gn_destroy": ([v], None),
        "gn_last_error": ([], C.c_char_p),
        "gn_volume": ([v], C.c_longlong),
        "gn_request_abort": ([v, C.c_int], None),
        "gn_selftest_wait_timeout": ([v], C.c_int),
        "gn_sigma_mass": ([v, _dp, _dp], C.c_int),
        "gn_dirac": ([v, _dp, _dp, _dp, C.c_int, C.c_int], C.c_int),
        "gn_cg": ([v, _dp, _dp, _dp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_longlong, C.c_int,
                   C.POINTER(CgInfo)], C.c_int),
        "gn_sigma_force": ([v, C.c_double, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp, C.c_int, C.POINTER(CgInfo)],
                           C.c_int),
        "gn_energy": ([v, C.c_double, _dp, _dp, _dp, _dp, _dp], C.c_int),
        "gn_evolve_sigma": ([v, _dp, _dp, _dp, C.c_double], C.c_int),
        "gn_evolve_momenta": ([v, _dp, _dp, C.c_double], C.c_int),
        "gn_condensate": ([v, _dp, C.c_double, _dp, _dp, C.c_void_p, _dp, _dp, C.POINTER(C.c_longlong), C.c_int],
                          C.c_int),
        "gn_load_sigma": ([v, _dp], C.c_int),
        "gn_store_sigma": ([v, _dp, _dp], C.c_int),
        "gn_read_state": ([v, C.c_int, _dp], C.c_int),
        "gn_write_state": ([v, C.c_int, _dp], C.c_int),
        "gn_trajectory": ([v, C.POINTER(HmcParams), C.c_void_p, C.c_void_p, C.POINTER(TrajResult)], C.c_int),
        "gn_stream": ([v], C.c_void_p),
        "gn_field_ptr": ([v, C.c_int], C.c_void_p),
        "gn_dirac_device": ([v, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int], C.c_int),
        "gn_cg_device": ([v, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                          C.c_longlong, C.c_int, C.POINTER(CgInfo)], C.c_int),
        "gn_trajectory_device": ([v, C.POINTER(HmcParams), C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(TrajResult)], C.c_int),
        "gn_md_evolve": ([v, C.POINTER(HmcParams), C.POINTER(TrajResult)], C.c_int),
        "gn_evolve_sigma_in_time": ([v, C.POINTER(HmcParams), C.POINTER(TrajResult)], C.c_int),
        "gn_launch_count": ([v], C.c_longlong),
        "gn_flush_l2": ([v], C.c_int),
        "gn_set_parity_mode": ([v, C.c_int], C.c_int),
        "gn_set_reliable_interval": ([v, C.c_int], C.c_int),
        "gn_ensemble_create": ([C.POINTER(v), C.c_int, C.POINTER(C.c_int), _dp, C.POINTER(C.c_ulonglong),
                                C.c_ulonglong, C.c_int], C.c_int),
        "gn_ensemble_destroy": ([v], None),
        "gn_ensemble_load_sigma": ([v, C.c_int, _dp], C.c_int),
        "gn_ensemble_store_sigma": ([v, C.c_int, _dp, _dp], C.c_int),
        "gn_ensemble_set_layout": ([v, C.c_int, C.c_longlong], C.c_int),
        "gn_ensemble_tune": ([v, C.POINTER(EnsParams), C.POINTER(C.c_int), C.POINTER(C.c_longlong)], C.c_int),
        "gn_ensemble_run": ([v, C.POINTER(EnsParams), C.c_int, C.c_int], C.c_int),
        "gn_ensemble_stats": ([v, C.POINTER(ChainStats), C.c_int], C.c_int),
        "gn_ensemble_stream": ([v], C.c_void_p),
        "gn_server_create": ([C.POINTER(v), C.POINTER(EnsParams), C.c_double, C.c_ulonglong, C.c_int,
                              C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.c_int], C.c_int),
        "gn_server_destroy": ([v], None),
        "gn_server_add_chain": ([v, C.c_int, C.c_double, _dp, C.c_ulonglong], C.c_int),
        "gn_server_clock": ([v], C.c_double),
        "gn_server_submit": ([v, C.c_int, C.c_int, C.c_int, C.c_double], C.c_longlong),
        "gn_server_step": ([v, C.POINTER(C.c_int)], C.c_int),
        "gn_server_request": ([v, C.c_longlong, C.POINTER(ReqInfo)], C.c_int),
        "gn_server_solution": ([v, C.c_longlong, _dp], C.c_int),
        "gn_server_chain_sigma": ([v, C.c_int, _dp], C.c_int),
        "gn_server_load": ([v, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong)], C.c_int),
        "gn_ensemble_info": ([v, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                              C.POINTER(C.c_int)], C.c_int),
        "gn_condensate_sigma": ([v, _dp, _dp], C.c_int),
        "gn_condensate_sigma_device": ([v, C.c_void_p, _dp], C.c_int),
        "gn_checkpoint_write_file": ([C.c_char_p, C.c_char_p, C.c_int, _dp, _dp, _dp, C.POINTER(HmcCounters)],
                                     C.c_int),
        "gn_checkpoint_read_file": ([C.c_char_p, C.c_int, _dp, _dp, C.POINTER(HmcCounters), _dp], C.c_int),
        "gn_checkpoint_check_value": ([C.c_int, _dp, _dp], C.c_double),
        "gn_checkpoint_save": ([v, C.c_char_p, C.c_char_p, C.POINTER(HmcCounters)], C.c_int),
        "gn_checkpoint_load": ([v, C.c_char_p, C.c_char_p, C.POINTER(HmcCounters)], C.c_int),
        "gn_ensemble_observables": ([v, _dp], C.c_int),
        "gn_ensemble_set_autoregulation": ([v, C.c_int, C.c_int], C.c_int),
        "gn_ensemble_checkpoint_save": ([v, C.c_int, C.c_char_p, C.c_char_p, C.POINTER(HmcCounters)], C.c_int),
        "gn_ensemble_checkpoint_load": ([v, C.c_int, C.c_char_p, C.c_char_p, C.POINTER(HmcCounters)], C.c_int),
        "gn_format_measure_line": ([C.c_char_p, C.c_size_t, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _dp, _dp], C.c_int),
        "gn_load_pi": ([v, _dp], C.c_int),
        "gn_store_pi": ([v, _dp, _dp], C.c_int),
        "gn_set_u1": ([v, C.c_int], C.c_int),
        "gn_dirac_u1": ([v, _dp, _dp, _dp, _dp, C.c_int, C.c_int], C.c_int),
        "gn_cg_u1": ([v, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int, C.c_int, C.c_longlong, C.c_int,
                      C.POINTER(CgInfo)],
                     C.c_int),
        "gn_sigma_force_u1": ([v, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp, C.POINTER(CgInfo)],
                              C.c_int),
        "gn_pi_force": ([v, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp, C.POINTER(CgInfo)], C.c_int),
        "gn_energy_u1": ([v, C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp], C.c_int),
        "gn_trajectory_pi": ([v, C.POINTER(HmcParams), C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(TrajResult)],
                             C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _path(p):
    return None if p is None else str(p).encode()


def _raise(st):
    raise GnError(st, load_library().gn_last_error().decode())


# ---- the reference's lattice file (host functions, no device needed)
def checkpoint_write_file(path, path_copy, L, sigma, sigmamass, counters, links=None):
    """WriteBinaryLattice's file (simulation.c:129-185): links None = unit links."""
    lib = load_library()
    s = np.ascontiguousarray(sigma, np.float64)
    sm = np.ascontiguousarray(sigmamass, np.float64)
    lk = None if links is None else _p(np.ascontiguousarray(links, np.float64))
    c = counters if isinstance(counters, HmcCounters) else HmcCounters.from_dict(counters)
    st = lib.gn_checkpoint_write_file(_path(path), _path(path_copy), int(L), _p(s), _p(sm), lk, C.byref(c))
    if st != GN_OK:
        _raise(st)


def checkpoint_read_file(path, L):
    """One lattice file: (sigma, links (V, 3, 2), counters dict, stored check value)."""
    lib = load_library()
    V = int(L) ** 3
    s, lk, chk = np.empty(V), np.empty(6 * V), C.c_double()
    c = HmcCounters()
    st = lib.gn_checkpoint_read_file(_path(path), int(L), _p(s), _p(lk), C.byref(c), C.byref(chk))
    if st != GN_OK:
        _raise(st)
    return s, lk.reshape(V, 3, 2), c.as_dict(), chk.value


def checkpoint_check_value(L, sigmamass, links=None):
    """TestWriteReadLattice (simulation.c:101-120) of (sigmamass, links)."""
    sm = np.ascontiguousarray(sigmamass, np.float64)
    lk = None if links is None else _p(np.ascontiguousarray(links, np.float64))
    return load_library().gn_checkpoint_check_value(int(L), _p(sm), lk)


def format_measure_line(measure, L, beta, beta_scalar, mass, avg_iterations, avg_distance, cond_dirac=None,
                        cond_sigma=None):
    """TakeMeasures' observables line (observables.c:266-292)."""
    lib = load_library()
    cd = None if cond_dirac is None else _p(np.ascontiguousarray(cond_dirac, np.float64))
    cs = None if cond_sigma is None else _p(np.ascontiguousarray(cond_sigma, np.float64))
    n = lib.gn_format_measure_line(None, 0, measure, L, beta, beta_scalar, mass, avg_iterations, avg_distance, cd, cs)
    buf = C.create_string_buffer(n + 1)
    lib.gn_format_measure_line(buf, n + 1, measure, L, beta, beta_scalar, mass, avg_iterations, avg_distance, cd, cs)
    return buf.value.decode()


def _planes(a) -> tuple[np.ndarray, int]:
    """complex -> (re, im) planes; real -> itself."""
    if np.iscomplexobj(a):
        return np.ascontiguousarray(np.concatenate([a.real, a.imag]), np.float64), 2
    return np.ascontiguousarray(a, np.float64), 1


def _unplanes(a: np.ndarray, nc: int, V: int):
    return a[:V] + 1j * a[V:] if nc == 2 else a


def fn_address(f) -> int | None:
    """Address of a C function for the random-number hooks: accepts an int, a
    ctypes function pointer or a Python callable (wrapped; keep a reference)."""
    if f is None:
        return None
    if isinstance(f, int):
        return f
    if isinstance(f, C._CFuncPtr):
        return C.cast(f, C.c_void_p).value
    cb = DRAW_FN(f)
    _keepalive.append(cb)
    return C.cast(cb, C.c_void_p).value


_keepalive: list = []


class Lattice:
    """A device-resident L^3 lattice (one gn_context)."""

    def __init__(self, L: int, device: int = 0):
        self.lib = load_library()
        self.ctx = C.c_void_p()
        self._check(self.lib.gn_create(C.byref(self.ctx), L, device))
        self.L = L
        self.V = L ** 3

    def close(self):
        if self.ctx:
            self.lib.gn_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int, allow=(GN_OK,)):
        if st not in allow:
            raise GnError(st, self.lib.gn_last_error().decode())
        return st

    # ---- operators
    def sigma_mass(self, sigma):
        s = np.ascontiguousarray(sigma, np.float64)
        sm = np.empty(self.V)
        self._check(self.lib.gn_sigma_mass(self.ctx, _p(s), _p(sm)))
        return sm

    def dirac(self, sm, psi, op=GN_OP_M, out=None):
        inp, nc = _planes(psi)
        if op == GN_OP_SUB_M:
            o, _ = _planes(out)
            o = o.copy()
        else:
            o = np.zeros_like(inp)
        self._check(self.lib.gn_dirac(self.ctx, _p(np.ascontiguousarray(sm, np.float64)), _p(inp), _p(o), nc, op))
        return _unplanes(o, nc, self.V)

    def cg(self, sm, b, x0=None, tol=1e-9, variant=0, relative=False, max_iter=0, precision=GN_PREC_FP64):
        """Solve (M M^T) x = b.  b: (V,) or (nrhs, V), real or complex.  Returns (x, infos, status)."""
        b = np.asarray(b)
        single = b.ndim == 1
        bb = b[None] if single else b
        nrhs = bb.shape[0]
        cplx = np.iscomplexobj(bb) or (x0 is not None and np.iscomplexobj(x0))
        nc = 2 if cplx else 1
        if cplx:
            bb = bb.astype(np.complex128)
            bp = np.concatenate([np.concatenate([r.real, r.imag]) for r in bb])
        else:
            bp = bb.astype(np.float64).reshape(-1)
        if x0 is None:
            xp = np.zeros_like(bp)
        else:
            xx = np.asarray(x0)
            xx = xx[None] if xx.ndim == 1 else xx
            xp = (np.concatenate([np.concatenate([r.real, r.imag]) for r in xx.astype(np.complex128)]) if cplx
                  else xx.astype(np.float64).reshape(-1))
        bp = np.ascontiguousarray(bp)
        xp = np.ascontiguousarray(xp, np.float64).copy()
        infos = (CgInfo * nrhs)()
        st = self._check(self.lib.gn_cg(self.ctx, _p(np.ascontiguousarray(sm, np.float64)), _p(bp), _p(xp), nrhs,
                                        nc, tol, variant, int(relative), max_iter, precision, infos),
                         allow=(GN_OK, GN_NOT_CONVERGED))
        V = self.V
        xs = [_unplanes(xp[k * nc * V:(k + 1) * nc * V], nc, V) for k in range(nrhs)]
        x = xs[0] if single else np.stack(xs)
        return x, [i.as_dict() for i in infos], st

    def sigma_force(self, beta_s, sigma, sm, phi, X, tol, precision=GN_PREC_FP64):
        phi = np.ascontiguousarray(phi, np.float64).reshape(-1)
        Xp = np.array(X, np.float64).reshape(-1)
        Y = np.zeros(2 * self.V)
        F = np.zeros(self.V)
        infos = (CgInfo * 2)()
        st = self._check(self.lib.gn_sigma_force(self.ctx, beta_s, _p(np.ascontiguousarray(sigma, np.float64)),
                                                 _p(np.ascontiguousarray(sm, np.float64)), _p(phi), _p(Xp), _p(Y),
                                                 tol, _p(F), precision, infos), allow=(GN_OK, GN_NOT_CONVERGED))
        return F, Xp.reshape(2, -1), Y.reshape(2, -1), [i.as_dict() for i in infos], st

    def energy(self, beta_s, sigma, P, phi, X):
        H = C.c_double()
        self._check(self.lib.gn_energy(self.ctx, beta_s, _p(np.ascontiguousarray(sigma, np.float64)),
                                       _p(np.ascontiguousarray(P, np.float64)),
                                       _p(np.ascontiguousarray(phi, np.float64).reshape(-1)),
                                       _p(np.ascontiguousarray(X, np.float64).reshape(-1)), C.byref(H)))
        return H.value

    def evolve_sigma(self, sigma, P, eps):
        s = np.array(sigma, np.float64)
        sm = np.empty(self.V)
        self._check(self.lib.gn_evolve_sigma(self.ctx, _p(s), _p(sm), _p(np.ascontiguousarray(P, np.float64)), eps))
        return s, sm

    def evolve_momenta(self, P, F, eps):
        p = np.array(P, np.float64)
        self._check(self.lib.gn_evolve_momenta(self.ctx, _p(p), _p(np.ascontiguousarray(F, np.float64)), eps))
        return p

    def condensate(self, sm, tol, target, uniform, precision=GN_PREC_FP64):
        t = np.concatenate([np.real(target), np.imag(target)]).astype(np.float64)
        D = np.zeros(2 * self.V)
        out = np.zeros(11)
        it = C.c_double()
        calls = C.c_longlong()
        st = self._check(self.lib.gn_condensate(self.ctx, _p(np.ascontiguousarray(sm, np.float64)), tol, _p(t), _p(D),
                                                fn_address(uniform), _p(out), C.byref(it), C.byref(calls), precision),
                         allow=(GN_OK, GN_NOT_CONVERGED))
        V = self.V
        return out, t[:V] + 1j * t[V:], D[:V] + 1j * D[V:], it.value, calls.value, st

    # ---- resident state
    def load_sigma(self, sigma):
        self._check(self.lib.gn_load_sigma(self.ctx, _p(np.ascontiguousarray(sigma, np.float64))))

    def store_sigma(self):
        s = np.empty(self.V)
        sm = np.empty(self.V)
        self._check(self.lib.gn_store_sigma(self.ctx, _p(s), _p(sm)))
        return s, sm

    def read_state(self, field):
        if field in (GN_F_P, GN_F_F, GN_F_PI_P, GN_F_PI_F):
            n = self.V
        elif field in (GN_F_CHI_C, GN_F_PHI_C, GN_F_X_C, GN_F_Y_C):
            n = 4 * self.V
        else:
            n = 2 * self.V
        a = np.empty(n)
        self._check(self.lib.gn_read_state(self.ctx, field, _p(a)))
        return a if n == self.V else a.reshape(n // self.V, self.V)

    def write_state(self, field, a):
        self._check(self.lib.gn_write_state(self.ctx, field, _p(np.ascontiguousarray(a, np.float64).reshape(-1))))

    def trajectory(self, beta_s, eps, steps, gauss=None, uniform=None, integrator=GN_LFMN2VF, tol_medium=1e-3,
                   tol_high=1e-9, relative=False, precision=GN_PREC_FP64):
        hp = HmcParams(beta_s, eps, steps, integrator, tol_medium, tol_high, int(relative), precision)
        res = TrajResult()
        self._check(self.lib.gn_trajectory(self.ctx, C.byref(hp), fn_address(gauss), fn_address(uniform),
                                           C.byref(res)), allow=(GN_OK, GN_NOT_CONVERGED))
        return res.as_dict()

    def md_evolve(self, beta_s, eps, steps, integrator=GN_LFMN2VF, tol_medium=1e-3, tol_high=1e-9, relative=False,
                  precision=GN_PREC_FP64):
        """The MD of one trajectory on the resident sigma, P and phi, without
        draws or Metropolis test (the reference's EvolveSigmaInTime* helpers)."""
        hp = HmcParams(beta_s, eps, steps, integrator, tol_medium, tol_high, int(relative), precision)
        res = TrajResult()
        self._check(self.lib.gn_md_evolve(self.ctx, C.byref(hp), C.byref(res)), allow=(GN_OK, GN_NOT_CONVERGED))
        return res.as_dict()

    def evolve_in_time(self, beta_s, eps, steps, integrator=GN_LFMN2VF, tol_medium=1e-3, tol_high=1e-9,
                       relative=False, precision=GN_PREC_FP64):
        """The reference's EvolveSigmaInTime* helper of `integrator` on the
        resident sigma, P, phi and X (gn_evolve_sigma_in_time)."""
        hp = HmcParams(beta_s, eps, steps, integrator, tol_medium, tol_high, int(relative), precision)
        res = TrajResult()
        self._check(self.lib.gn_evolve_sigma_in_time(self.ctx, C.byref(hp), C.byref(res)),
                    allow=(GN_OK, GN_NOT_CONVERGED))
        return res.as_dict()

    def set_parity_mode(self, on=True):
        """M^T and the energy in the reference's exact order (see GN_PREC_FP64_EXACT)."""
        self._check(self.lib.gn_set_parity_mode(self.ctx, int(on)))

    def set_reliable_interval(self, n):
        """Mixed precision: a reliable update at least every n inner iterations."""
        self._check(self.lib.gn_set_reliable_interval(self.ctx, int(n)))

    def request_abort(self, on=True):
        self.lib.gn_request_abort(self.ctx, int(on))

    def selftest_wait_timeout(self):
        """Status of the failure-detection self-test (GN_ERR_TIMEOUT when the bounded wait works)."""
        return self.lib.gn_selftest_wait_timeout(self.ctx)

    # ---- device-resident entry points (pointers are ints)
    @property
    def stream(self) -> int:
        return self.lib.gn_stream(self.ctx)

    def field_ptr(self, field) -> int:
        return self.lib.gn_field_ptr(self.ctx, field)

    def dirac_device(self, sm_ptr, in_ptr, out_ptr, ncomp=1, op=GN_OP_M):
        self._check(self.lib.gn_dirac_device(self.ctx, sm_ptr, in_ptr, out_ptr, ncomp, op))

    def cg_device(self, sm_ptr, b_ptr, x_ptr, nrhs, ncomp=1, tol=1e-9, variant=1, relative=False, max_iter=0,
                  precision=GN_PREC_FP64):
        infos = (CgInfo * nrhs)()
        st = self._check(self.lib.gn_cg_device(self.ctx, sm_ptr, b_ptr, x_ptr, nrhs, ncomp, tol, variant,
                                               int(relative), max_iter, precision, infos),
                         allow=(GN_OK, GN_NOT_CONVERGED))
        return [i.as_dict() for i in infos], st

    def trajectory_device(self, P_ptr, chi_ptr, beta_s, eps, steps, uniform=None, integrator=GN_LFMN2VF,
                          tol_medium=1e-3, tol_high=1e-9, relative=False, precision=GN_PREC_FP64):
        hp = HmcParams(beta_s, eps, steps, integrator, tol_medium, tol_high, int(relative), precision)
        res = TrajResult()
        self._check(self.lib.gn_trajectory_device(self.ctx, C.byref(hp), P_ptr, chi_ptr, fn_address(uniform),
                                                  C.byref(res)), allow=(GN_OK, GN_NOT_CONVERGED))
        return res.as_dict()

    def launch_count(self) -> int:
        return self.lib.gn_launch_count(self.ctx)

    def flush_l2(self):
        self._check(self.lib.gn_flush_l2(self.ctx))

    # ---- the U(1) model (complex fields as numpy complex128, shape (nsys, V))
    @staticmethod
    def _cplanes(a):
        a = np.asarray(a, np.complex128)
        a = a[None] if a.ndim == 1 else a
        return np.ascontiguousarray(np.concatenate([np.concatenate([r.real, r.imag]) for r in a])), a.shape[0]

    def _uncplanes(self, p, n):
        p = p.reshape(n, 2, self.V)
        return p[:, 0] + 1j * p[:, 1]

    def load_pi(self, pi):
        """The resident pi (and pimass); the context switches to the U(1) model."""
        self._check(self.lib.gn_load_pi(self.ctx, _p(np.ascontiguousarray(pi, np.float64))))

    def store_pi(self):
        pi, pm = np.empty(self.V), np.empty(self.V)
        self._check(self.lib.gn_store_pi(self.ctx, _p(pi), _p(pm)))
        return pi, pm

    def set_u1(self, on=True):
        self._check(self.lib.gn_set_u1(self.ctx, int(on)))

    def dirac_u1(self, sm, pm, psi, op=GN_OP_M, out=None):
        """M, M^dagger or out - M psi with the complex mass; psi complex (V,) or (nsys, V)."""
        single = np.asarray(psi).ndim == 1
        inp, n = self._cplanes(psi)
        o = self._cplanes(out)[0].copy() if op == GN_OP_SUB_M else np.zeros_like(inp)
        self._check(self.lib.gn_dirac_u1(self.ctx, _p(np.ascontiguousarray(sm, np.float64)),
                                         _p(np.ascontiguousarray(pm, np.float64)), _p(inp), _p(o), n, op))
        r = self._uncplanes(o, n)
        return r[0] if single else r

    def cg_u1(self, sm, pm, b, x0=None, tol=1e-9, variant=0, relative=False, max_iter=0, precision=GN_PREC_FP64):
        single = np.asarray(b).ndim == 1
        bp, n = self._cplanes(b)
        xp = np.zeros_like(bp) if x0 is None else self._cplanes(x0)[0].copy()
        infos = (CgInfo * n)()
        st = self._check(self.lib.gn_cg_u1(self.ctx, _p(np.ascontiguousarray(sm, np.float64)),
                                           _p(np.ascontiguousarray(pm, np.float64)), _p(bp), _p(xp), n, tol,
                                           variant, int(relative), max_iter, precision, infos),
                         allow=(GN_OK, GN_NOT_CONVERGED))
        x = self._uncplanes(xp, n)
        return (x[0] if single else x), [i.as_dict() for i in infos], st

    def _force_u1(self, fn, beta_s, fld, sm, pm, phi, X, tol):
        php, _ = self._cplanes(phi)
        Xp = self._cplanes(X)[0].copy()
        Y = np.zeros(4 * self.V)
        F = np.zeros(self.V)
        infos = (CgInfo * 2)()
        st = self._check(fn(self.ctx, beta_s, _p(np.ascontiguousarray(fld, np.float64)),
                            _p(np.ascontiguousarray(sm, np.float64)), _p(np.ascontiguousarray(pm, np.float64)),
                            _p(php), _p(Xp), _p(Y), tol, _p(F), infos), allow=(GN_OK, GN_NOT_CONVERGED))
        return F, self._uncplanes(Xp, 2), self._uncplanes(Y, 2), [i.as_dict() for i in infos], st

    def sigma_force_u1(self, beta_s, sigma, sm, pm, phi, X, tol):
        """ComputeSigmaForce in the U(1) model: (F, X, Y, infos, status); phi, X complex (2, V)."""
        return self._force_u1(self.lib.gn_sigma_force_u1, beta_s, sigma, sm, pm, phi, X, tol)

    def pi_force(self, beta_s, pi, sm, pm, phi, X, tol):
        """ComputePiForce: (F, X, Y, infos, status); phi, X complex (2, V)."""
        return self._force_u1(self.lib.gn_pi_force, beta_s, pi, sm, pm, phi, X, tol)

    def energy_u1(self, which, beta_s, field, P, phi, X):
        """which 0: ComputeFullEnergyForSigma, 1: ComputeFullEnergyForPi (phi, X complex (2, V))."""
        H = C.c_double()
        self._check(self.lib.gn_energy_u1(self.ctx, which, beta_s, _p(np.ascontiguousarray(field, np.float64)),
                                          _p(np.ascontiguousarray(P, np.float64)), _p(self._cplanes(phi)[0]),
                                          _p(self._cplanes(X)[0]), C.byref(H)))
        return H.value

    def trajectory_pi(self, beta_s, eps, steps, gauss_pair=None, gauss=None, uniform=None, tol_high=1e-9,
                      relative=False, precision=GN_PREC_FP64):
        """LeapFrog2Pi on the resident sigma and pi.  gauss_pair(a, b) fills two
        N(0, 1) values (the reference's Gauss2MeanVariance(a, b, 0, 1)): an int
        address, a PAIR_FN or a Python callable taking two POINTER(c_double)."""
        hp = HmcParams(beta_s, eps, steps, 0, tol_high, tol_high, int(relative), precision)
        res = TrajResult()
        if gauss_pair is not None and not isinstance(gauss_pair, (int, C._CFuncPtr)):
            gauss_pair = PAIR_FN(gauss_pair)
        keep = gauss_pair  # the callback must outlive the call
        pair = None if gauss_pair is None else (gauss_pair if isinstance(gauss_pair, int)
                                                else C.cast(gauss_pair, C.c_void_p).value)
        self._check(self.lib.gn_trajectory_pi(self.ctx, C.byref(hp), pair, fn_address(gauss), fn_address(uniform),
                                              C.byref(res)), allow=(GN_OK, GN_NOT_CONVERGED))
        del keep
        return res.as_dict()

    # ---- observables and checkpoints
    def condensate_sigma(self, sigma=None):
        """CondensateSigmaPi of sigma (host array) or of the resident sigma (None)."""
        out = np.empty(8)
        s = None if sigma is None else _p(np.ascontiguousarray(sigma, np.float64))
        self._check(self.lib.gn_condensate_sigma(self.ctx, s, _p(out)))
        return out

    def checkpoint_save(self, path, path_copy, counters):
        c = counters if isinstance(counters, HmcCounters) else HmcCounters.from_dict(counters)
        self._check(self.lib.gn_checkpoint_save(self.ctx, _path(path), _path(path_copy), C.byref(c)))

    def checkpoint_load(self, path, path_copy=None):
        """(status, counters): GN_OK, GN_ERR_NOT_FOUND (a fresh start) or GN_ERR_FORMAT."""
        c = HmcCounters()
        st = self._check(self.lib.gn_checkpoint_load(self.ctx, _path(path), _path(path_copy), C.byref(c)),
                         allow=(GN_OK, GN_ERR_NOT_FOUND, GN_ERR_FORMAT))
        return st, c.as_dict()


class Ensemble:
    """Many independent sigma-HMC chains (gn_ensemble_* of gn_b200.h)."""

    def __init__(self, Ls, betas, seed=1231, stream_ids=None, device=0):
        self.lib = load_library()
        self.Ls = [int(x) for x in Ls]
        self.n = len(self.Ls)
        Larr = (C.c_int * self.n)(*self.Ls)
        barr = np.ascontiguousarray(betas, np.float64)
        ids = None if stream_ids is None else (C.c_ulonglong * self.n)(*[int(x) for x in stream_ids])
        self.ens = C.c_void_p()
        self._check(self.lib.gn_ensemble_create(C.byref(self.ens), self.n, Larr, _p(barr), ids, int(seed), device))

    def _check(self, st, allow=(GN_OK,)):
        if st not in allow:
            raise GnError(st, self.lib.gn_last_error().decode())
        return st

    def close(self):
        if self.ens:
            self.lib.gn_ensemble_destroy(self.ens)
            self.ens = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def load_sigma(self, c, sigma):
        s = np.ascontiguousarray(sigma, np.float64)
        assert s.size == self.Ls[c] ** 3
        self._check(self.lib.gn_ensemble_load_sigma(self.ens, c, _p(s)))

    def store_sigma(self, c):
        V = self.Ls[c] ** 3
        s, sm = np.empty(V), np.empty(V)
        self._check(self.lib.gn_ensemble_store_sigma(self.ens, c, _p(s), _p(sm)))
        return s, sm

    @staticmethod
    def params(eps, steps, integrator=GN_LFMN2VF, tol=1e-10, precision=GN_PREC_MIXED):
        return EnsParams(eps, steps, integrator, tol, precision)

    def set_layout(self, group_blocks, big_min_volume):
        self._check(self.lib.gn_ensemble_set_layout(self.ens, group_blocks, big_min_volume))

    def tune(self, p):
        gs, vmin = C.c_int(), C.c_longlong()
        self._check(self.lib.gn_ensemble_tune(self.ens, C.byref(p), C.byref(gs), C.byref(vmin)))
        return gs.value, vmin.value

    def run(self, p, ntraj, graph=True):
        self._check(self.lib.gn_ensemble_run(self.ens, C.byref(p), int(ntraj), int(graph)))

    def stats(self, reset=False):
        out = (ChainStats * self.n)()
        self._check(self.lib.gn_ensemble_stats(self.ens, out, int(reset)))
        return [o.as_dict() for o in out]

    @property
    def stream(self):
        """The cudaStream_t (as an int) the ensemble runs on."""
        return self.lib.gn_ensemble_stream(self.ens)

    def observables(self):
        """(nchains, 8): per-chain means of CondensateSigmaPi's outputs over the
        trajectories since the last stats reset."""
        out = np.empty(8 * self.n)
        self._check(self.lib.gn_ensemble_observables(self.ens, _p(out)))
        return out.reshape(self.n, 8)

    def set_autoregulation(self, on=True, chain=-1):
        """UpdateHMCParameters per chain after every trajectory (chain -1: all)."""
        self._check(self.lib.gn_ensemble_set_autoregulation(self.ens, int(chain), int(on)))

    def checkpoint_save(self, c, path, path_copy=None, counters=None):
        """counters None: the chain's own (accepted, done, story)."""
        if counters is None:
            cnt = None
        else:
            cnt = C.byref(counters if isinstance(counters, HmcCounters) else HmcCounters.from_dict(counters))
        self._check(self.lib.gn_ensemble_checkpoint_save(self.ens, c, _path(path), _path(path_copy), cnt))

    def checkpoint_load(self, c, path, path_copy=None):
        cnt = HmcCounters()
        st = self._check(self.lib.gn_ensemble_checkpoint_load(self.ens, c, _path(path), _path(path_copy),
                                                              C.byref(cnt)),
                         allow=(GN_OK, GN_ERR_NOT_FOUND, GN_ERR_FORMAT))
        return st, cnt.as_dict()

    def info(self):
        gs, vmin, g, nl = C.c_int(), C.c_longlong(), C.c_int(), C.c_int()
        self._check(self.lib.gn_ensemble_info(self.ens, C.byref(gs), C.byref(vmin), C.byref(g), C.byref(nl)))
        return {"group_blocks": gs.value, "big_min_volume": vmin.value, "graph": g.value,
                "launches_per_trajectory": nl.value}


class Server:
    """Requests on resident chains with continuous batching (gn_server_* of gn_b200.h)."""

    # Team tiers: L >= 32 shares the whole GPU (teams of at least 32 blocks),
    # L = 16..24 runs on 8 blocks, L = 12 on 2, the rest on single blocks.
    # Measured with bench.py's serving mix at 50 requests/s: p50 54 ms, p99
    # 454 ms, against 154 ms and 1.3 s for the older ((16, 48^3), (4, 16^3)),
    # which left L = 32 and 40 on teams of 4 blocks (80 and 148 ms for one
    # trajectory alone, against 55-68 ms for L = 48-64 on the whole GPU); a
    # step lasts as long as its costliest slice, so those slices held up every
    # request beside them.
    DEFAULT_TIERS = ((32, 32 ** 3), (8, 16 ** 3), (2, 12 ** 3))

    def __init__(self, traj_params, mem_budget_bytes=8e9, seed=1231, tiers=DEFAULT_TIERS, device=0):
        """tiers: (blocks per team, minimum volume) pairs, team sizes dividing each other."""
        self.lib = load_library()
        self.srv = C.c_void_p()
        nt = len(tiers)
        tb = (C.c_int * max(nt, 1))(*[int(t[0]) for t in tiers])
        tv = (C.c_longlong * max(nt, 1))(*[int(t[1]) for t in tiers])
        self._check(self.lib.gn_server_create(C.byref(self.srv), C.byref(traj_params), float(mem_budget_bytes),
                                              int(seed), nt, tb, tv, device))
        self.Ls = []

    def _check(self, st, allow=(GN_OK,)):
        if st not in allow:
            raise GnError(st, self.lib.gn_last_error().decode())
        return st

    def close(self):
        if self.srv:
            self.lib.gn_server_destroy(self.srv)
            self.srv = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_chain(self, L, beta_s, sigma, stream_id):
        s = np.ascontiguousarray(sigma, np.float64)
        c = self.lib.gn_server_add_chain(self.srv, int(L), float(beta_s), _p(s), int(stream_id))
        if c < 0:
            raise GnError(c, self.lib.gn_last_error().decode())
        self.Ls.append(int(L))
        return c

    def clock(self):
        return self.lib.gn_server_clock(self.srv)

    def submit(self, chain, rtype, noise_vectors=0, t_arrival=None):
        t = self.clock() if t_arrival is None else float(t_arrival)
        rid = self.lib.gn_server_submit(self.srv, int(chain), int(rtype), int(noise_vectors), t)
        if rid < 0:
            raise GnError(int(rid), self.lib.gn_last_error().decode())
        return rid

    def step(self):
        n = C.c_int()
        self._check(self.lib.gn_server_step(self.srv, C.byref(n)))
        return n.value

    def request(self, rid):
        r = ReqInfo()
        self._check(self.lib.gn_server_request(self.srv, int(rid), C.byref(r)))
        return r.as_dict()

    def solution(self, rid):
        info = self.request(rid)
        x = np.empty(self.Ls[info["chain"]] ** 3)
        self._check(self.lib.gn_server_solution(self.srv, int(rid), _p(x)))
        return x

    def chain_sigma(self, c):
        s = np.empty(self.Ls[c] ** 3)
        self._check(self.lib.gn_server_chain_sigma(self.srv, int(c), _p(s)))
        return s

    def load(self):
        r, q, b = C.c_int(), C.c_int(), C.c_longlong()
        self._check(self.lib.gn_server_load(self.srv, C.byref(r), C.byref(q), C.byref(b)))
        return {"running": r.value, "queued": q.value, "bytes_in_use": b.value}

    def drain(self, max_steps=100000):
        """Steps until nothing is running or queued."""
        for _ in range(max_steps):
            ld = self.load()
            if ld["running"] == 0 and ld["queued"] == 0:
                return
            self.step()
        raise RuntimeError("server did not drain")
