"""ctypes front-ends of the two CPU oracles -- TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg import
this module, and only as the checker.

* :class:`Port` wraps ``gn_oracle.c`` (this repository's restatement of the
  reference's algorithm, run-time L, real arrays).  It builds itself with gcc
  on first use, so it also works on a machine without the reference tree.
* :class:`Ref` wraps ``ref_harness.c`` linked with the reference's own sources
  (one shared object per L, built by build_ref.py into oracle/_ref/).

Fields are float64 numpy arrays in the reference's fermion order
(lexicographic (x0*L + x1)*L + x2 with x2 = time fastest; even sites first).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_SRC = HERE / "gn_oracle.c"
PORT_LIB = HERE / "libgn_oracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)
DRAW_FN = C.CFUNCTYPE(C.c_double)

# op codes of gno_schedule (gn_oracle.c)
OP_F_MED, OP_F_HIGH, OP_P, OP_Q, OP_S_HIGH = 1, 2, 3, 4, 5


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def build_port(force: bool = False) -> Path:
    """Compile gn_oracle.c (no FMA contraction, like the reference's x86-64 build)."""
    if PORT_LIB.exists() and not force and PORT_LIB.stat().st_mtime >= PORT_SRC.stat().st_mtime:
        return PORT_LIB
    tmp = PORT_LIB.with_suffix(f".{os.getpid()}.tmp")
    subprocess.run(["gcc", "-O3", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(tmp), str(PORT_SRC), "-lm"],
                   check=True)
    os.replace(tmp, PORT_LIB)
    return PORT_LIB


def volume(L: int) -> int:
    return L * L * L


class Port:
    """The CPU restatement (gn_oracle.c)."""

    def __init__(self):
        self.lib = C.CDLL(str(build_port()))
        lib = self.lib
        lib.gno_sigma_mass.argtypes = [C.c_int, _dp, _dp]
        lib.gno_dirac.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_int]
        lib.gno_cg.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int, C.c_long, _lp, _ip]
        lib.gno_force.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, _lp]
        lib.gno_energy.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp]
        lib.gno_energy.restype = C.c_double
        lib.gno_evolve_sigma.argtypes = [C.c_int, _dp, _dp, _dp, C.c_double]
        lib.gno_evolve_momenta.argtypes = [C.c_int, _dp, _dp, C.c_double]
        lib.gno_schedule.argtypes = [C.c_int, C.c_double, C.c_int, _ip, _dp, C.c_int]
        lib.gno_trajectory.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double,
                                       _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_void_p, C.c_void_p, _dp, _dp,
                                       _lp, _dp]
        lib.gno_condensate.argtypes = [C.c_int, _dp, C.c_double, _dp, _dp, C.c_void_p, _dp, _dp, _lp]
        lib.gno_replay_set.argtypes = [_dp, C.c_long, _dp, C.c_long]
        lib.gno_replay_pos.argtypes = [_lp, _lp]
        lib.gno_tables.argtypes = [C.c_int, _ip, _ip, C.c_void_p, C.c_void_p]
        self._replay_keep = None

    # --- geometry / fields
    def tables(self, L):
        V = volume(L)
        pp = np.zeros(3 * V, np.int32)
        mm = np.zeros(3 * V, np.int32)
        ep = np.zeros(3 * V, np.int8)
        em = np.zeros(3 * V, np.int8)
        self.lib.gno_tables(L, pp.ctypes.data_as(_ip), mm.ctypes.data_as(_ip), ep.ctypes.data, em.ctypes.data)
        return pp.reshape(V, 3), mm.reshape(V, 3), ep.reshape(V, 3), em.reshape(V, 3)

    def sigma_mass(self, L, sigma):
        sigma = np.ascontiguousarray(sigma, np.float64)
        sm = np.empty_like(sigma)
        self.lib.gno_sigma_mass(L, _p(sigma), _p(sm))
        return sm

    def dirac(self, L, sm, psi, which=0, out=None):
        """which 0 = M, 1 = M^T, 2 = out - M psi.  psi real (V,) or complex (V,)."""
        sm = np.ascontiguousarray(sm, np.float64)
        cplx = np.iscomplexobj(psi)
        V = volume(L)
        inp = np.concatenate([psi.real, psi.imag]) if cplx else np.ascontiguousarray(psi, np.float64)
        if which == 2:
            o = out
            o = np.concatenate([o.real, o.imag]) if cplx else np.array(o, np.float64)
        else:
            o = np.zeros_like(inp)
        inp = np.ascontiguousarray(inp)
        self.lib.gno_dirac(L, _p(sm), _p(inp), _p(o), 2 if cplx else 1, which)
        return (o[:V] + 1j * o[V:]) if cplx else o

    def cg(self, L, sm, b, x0=None, tol=1e-9, variant=0, max_iter=None):
        """Returns (x, converged, iterations, counted)."""
        V = volume(L)
        cplx = np.iscomplexobj(b) or np.iscomplexobj(x0)
        nc = 2 if cplx else 1
        bb = np.concatenate([np.real(b), np.imag(b)]) if cplx else np.array(b, np.float64)
        if x0 is None:
            xx = np.zeros(nc * V)
        else:
            xx = np.concatenate([np.real(x0), np.imag(x0)]) if cplx else np.array(x0, np.float64)
        bb = np.ascontiguousarray(bb, np.float64)
        xx = np.ascontiguousarray(xx, np.float64)
        it = C.c_long(0)
        cnt = C.c_int(0)
        ok = self.lib.gno_cg(L, _p(np.ascontiguousarray(sm, np.float64)), _p(bb), _p(xx), nc, tol, variant,
                             max_iter if max_iter is not None else V + 1, C.byref(it), C.byref(cnt))
        x = (xx[:V] + 1j * xx[V:]) if cplx else xx
        return x, bool(ok), it.value, bool(cnt.value)

    def force(self, L, beta_s, sigma, sm, phi, X, tol):
        """ComputeSigmaForce. phi, X: (2, V); X is the CG start (in/out). Returns F, X, Y, ok, iters, calls."""
        V = volume(L)
        phi = np.ascontiguousarray(phi, np.float64).reshape(2 * V)
        X = np.array(X, np.float64).reshape(2 * V)
        Y = np.zeros(2 * V)
        F = np.zeros(V)
        itacc = C.c_double(0.0)
        calls = C.c_long(0)
        ok = self.lib.gno_force(L, beta_s, _p(np.ascontiguousarray(sigma, np.float64)),
                                _p(np.ascontiguousarray(sm, np.float64)), _p(phi), _p(X), _p(Y), tol, _p(F),
                                C.byref(itacc), C.byref(calls))
        return F, X.reshape(2, V), Y.reshape(2, V), bool(ok), itacc.value, calls.value

    def energy(self, L, beta_s, sigma, P, phi, X):
        return self.lib.gno_energy(L, beta_s, _p(np.ascontiguousarray(sigma, np.float64)),
                                   _p(np.ascontiguousarray(P, np.float64)),
                                   _p(np.ascontiguousarray(phi, np.float64).reshape(-1)),
                                   _p(np.ascontiguousarray(X, np.float64).reshape(-1)))

    def evolve_sigma(self, L, sigma, P, eps):
        s = np.array(sigma, np.float64)
        sm = np.empty_like(s)
        self.lib.gno_evolve_sigma(L, _p(s), _p(sm), _p(np.ascontiguousarray(P, np.float64)), eps)
        return s, sm

    def evolve_momenta(self, L, P, F, eps):
        p = np.array(P, np.float64)
        self.lib.gno_evolve_momenta(L, _p(p), _p(np.ascontiguousarray(F, np.float64)), eps)
        return p

    def schedule(self, integrator, eps, steps):
        ops = np.zeros(1024, np.int32)
        coefs = np.zeros(1024)
        n = self.lib.gno_schedule(integrator, eps, steps, ops.ctypes.data_as(_ip), _p(coefs), 1024)
        return ops[:n].copy(), coefs[:n].copy()

    # --- RNG replay
    def replay(self, gauss_seq, unif_seq):
        g = np.ascontiguousarray(gauss_seq, np.float64)
        u = np.ascontiguousarray(unif_seq, np.float64)
        self._replay_keep = (g, u)
        self.lib.gno_replay_set(_p(g), len(g), _p(u), len(u))
        return (C.cast(self.lib.gno_replay_gauss, C.c_void_p).value,
                C.cast(self.lib.gno_replay_uniform, C.c_void_p).value)

    def replay_pos(self):
        a, b = C.c_long(0), C.c_long(0)
        self.lib.gno_replay_pos(C.byref(a), C.byref(b))
        return a.value, b.value

    def trajectory(self, L, beta_s, eps, steps, state, gauss_fn, unif_fn, integrator=0, tol_med=1e-3, tol_high=1e-9):
        """state: dict with sigma, sm, P, F (V) and chi, phi, X, Y (2, V), iterations, calls, distance; updated in place.
        Returns (ok, dH, accepted, H0, H1)."""
        out = np.zeros(4)
        itacc = C.c_double(state.get("iterations", 0.0))
        calls = C.c_long(state.get("calls", 0))
        dist = C.c_double(state.get("distance", 0.0))
        arrs = {k: np.ascontiguousarray(state[k], np.float64) for k in ("sigma", "sm", "P", "F", "chi", "phi", "X", "Y")}
        ok = self.lib.gno_trajectory(L, beta_s, eps, steps, integrator, tol_med, tol_high, _p(arrs["sigma"]),
                                     _p(arrs["sm"]), _p(arrs["P"]), _p(arrs["F"]), _p(arrs["chi"]), _p(arrs["phi"]),
                                     _p(arrs["X"]), _p(arrs["Y"]), gauss_fn, unif_fn, _p(out), C.byref(itacc),
                                     C.byref(calls), C.byref(dist))
        state.update(arrs)
        state["iterations"], state["calls"], state["distance"] = itacc.value, calls.value, dist.value
        return bool(ok), out[0], bool(out[1]), out[2], out[3]

    def condensate(self, L, sm, tol, target, unif_fn):
        """Returns (out11, target, D, ok, iterations, calls); target complex (V,) in/out."""
        V = volume(L)
        t = np.concatenate([np.real(target), np.imag(target)]).astype(np.float64)
        D = np.zeros(2 * V)
        out = np.zeros(11)
        itacc = C.c_double(0.0)
        calls = C.c_long(0)
        ok = self.lib.gno_condensate(L, _p(np.ascontiguousarray(sm, np.float64)), tol, _p(t), _p(D), unif_fn,
                                     _p(out), C.byref(itacc), C.byref(calls))
        return out, t[:V] + 1j * t[V:], D[:V] + 1j * D[V:], bool(ok), itacc.value, calls.value


class Ref:
    """The reference's own code at one lattice size (oracle/_ref/libgnref_L{L}_i{I}.so)."""

    def __init__(self, L: int, integrator: int = 0, build: bool = True, extra_defs: tuple = (), tag: str = ""):
        """extra_defs / tag: a variant build (e.g. other CG tolerances) under its own name."""
        from . import build_ref  # noqa: F401  (package-relative when imported as oracle.oracle)
        path = build_ref.lib_path(L, integrator, tag)
        if build and build_ref.available():
            path = build_ref.build(L, integrator, tuple(extra_defs), tag)
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (the reference tree is needed to build it)")
        # RTLD_LOCAL: several L's can be loaded side by side
        self.lib = C.CDLL(str(path), mode=C.RTLD_LOCAL)
        self.L = L
        self.V = volume(L)
        lib = self.lib
        lib.gnref_init.argtypes = [C.c_uint, C.c_double, C.c_double, C.c_int]
        for name in ("gnref_gauss1", "gnref_casuale", "gnref_energy", "gnref_distance_sigma"):
            getattr(lib, name).restype = C.c_double
        lib.gnref_set_sigma.argtypes = [_dp]
        lib.gnref_get_sigma.argtypes = [_dp]
        lib.gnref_get_sigmamass.argtypes = [_dp]
        lib.gnref_set_sigmamass.argtypes = [_dp]
        lib.gnref_set_momenta.argtypes = [_dp]
        lib.gnref_get_momenta.argtypes = [_dp]
        lib.gnref_get_force.argtypes = [_dp]
        lib.gnref_kit_set.argtypes = [C.c_int, C.c_int, C.c_void_p]
        lib.gnref_kit_get.argtypes = [C.c_int, C.c_int, C.c_void_p]
        lib.gnref_counters.argtypes = [_dp, _ip]
        lib.gnref_dirac.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.gnref_cg.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_int]
        lib.gnref_force.argtypes = [C.c_double]
        lib.gnref_evolve_sigma.argtypes = [C.c_double]
        lib.gnref_evolve_momenta.argtypes = [C.c_double]
        lib.gnref_trajectory.argtypes = [C.c_char_p, _ip]
        lib.gnref_evolve_in_time.argtypes = [C.c_int, C.c_double, C.c_int]
        lib.gnref_info.argtypes = [_ip, _ip, _dp]
        lib.gnref_condensate.argtypes = [C.c_double, _dp]
        lib.gnref_seed.argtypes = [C.c_uint]
        lib.gnref_condensate_sigma.argtypes = [_dp]
        lib.gnref_write_lattice.argtypes = [C.c_char_p, C.c_char_p, _dp, _ip]
        lib.gnref_read_lattice.argtypes = [C.c_char_p, C.c_char_p, _dp, _ip]
        lib.gnref_read_lattice.restype = C.c_double
        for name in ("gnref_set_pi", "gnref_get_pi", "gnref_get_pimass", "gnref_set_pi_momenta",
                     "gnref_get_pi_momenta", "gnref_get_pi_force"):
            getattr(lib, name).argtypes = [_dp]
        lib.gnref_set_pi_params.argtypes = [C.c_double, C.c_int]
        lib.gnref_energy_pi.restype = C.c_double
        lib.gnref_trajectory_pi.argtypes = [C.c_char_p, _ip]
        lib.gnref_gauss2.argtypes = [_dp, _dp]

    def init(self, seed=1231, beta_s=0.85, eps=0.2, steps=2):
        self.lib.gnref_init(seed, beta_s, eps, steps)

    def check_tables(self) -> int:
        return self.lib.gnref_check_tables()

    def gauss(self, n):
        return np.array([self.lib.gnref_gauss1() for _ in range(n)])

    def uniform(self, n):
        return np.array([self.lib.gnref_casuale() for _ in range(n)])

    def rng_save(self):
        """Keep a copy of the global dSFMT state (random.c:9), to replay the same draws."""
        self.lib.gnref_rng_save()

    def rng_restore(self):
        self.lib.gnref_rng_restore()

    def fn_ptrs(self):
        return (C.cast(self.lib.gnref_gauss1, C.c_void_p).value, C.cast(self.lib.gnref_casuale, C.c_void_p).value)

    def set_sigma(self, sigma):
        self.lib.gnref_set_sigma(_p(np.ascontiguousarray(sigma, np.float64)))

    def sigma(self):
        s = np.empty(self.V)
        self.lib.gnref_get_sigma(_p(s))
        return s

    def sigmamass(self):
        s = np.empty(self.V)
        self.lib.gnref_get_sigmamass(_p(s))
        return s

    def set_sigmamass(self, sm):
        self.lib.gnref_set_sigmamass(_p(np.ascontiguousarray(sm, np.float64)))

    def set_momenta(self, P):
        self.lib.gnref_set_momenta(_p(np.ascontiguousarray(P, np.float64)))

    def momenta(self):
        s = np.empty(self.V)
        self.lib.gnref_get_momenta(_p(s))
        return s

    def force_buf(self):
        s = np.empty(self.V)
        self.lib.gnref_get_force(_p(s))
        return s

    KIT = {"chi": 0, "phi": 1, "X": 2, "Y": 3, "D": 4}

    def kit_set(self, which, f, v):
        a = np.ascontiguousarray(v, np.complex128)
        self.lib.gnref_kit_set(self.KIT[which], f, a.ctypes.data)

    def kit_get(self, which, f):
        a = np.empty(self.V, np.complex128)
        self.lib.gnref_kit_get(self.KIT[which], f, a.ctypes.data)
        return a

    def counters(self):
        it = C.c_double(0)
        calls = C.c_int(0)
        self.lib.gnref_counters(C.byref(it), C.byref(calls))
        return it.value, calls.value

    def dirac(self, psi, which=0, out=None):
        a = np.ascontiguousarray(psi, np.complex128)
        o = np.zeros(self.V, np.complex128) if out is None else np.array(out, np.complex128)
        self.lib.gnref_dirac(a.ctypes.data, o.ctypes.data, which)
        return o

    def cg(self, b, x0=None, tol=1e-9, variant=0, f=0):
        bb = np.ascontiguousarray(b, np.complex128)
        x = np.zeros(self.V, np.complex128) if x0 is None else np.array(x0, np.complex128)
        ok = self.lib.gnref_cg(bb.ctypes.data, x.ctypes.data, tol, variant, f)
        return x, bool(ok)

    def force(self, tol):
        return bool(self.lib.gnref_force(tol))

    def energy(self):
        return self.lib.gnref_energy()

    def evolve_sigma(self, eps):
        self.lib.gnref_evolve_sigma(eps)

    def evolve_momenta(self, eps):
        self.lib.gnref_evolve_momenta(eps)

    def trajectory(self, accfile: str):
        """Runs one trajectory; returns (ok, accepted, dH parsed from the acceptance line)."""
        acc = C.c_int(0)
        ok = self.lib.gnref_trajectory(accfile.encode(), C.byref(acc))
        dH = None
        if ok:
            with open(accfile) as fh:
                last = fh.read().strip().splitlines()[-1]
            dH = float(last.split("\t")[11])
        return bool(ok), bool(acc.value), dH

    def evolve_in_time(self, which, eps, steps):
        """EvolveSigmaInTime* (which: 0 LFMN2VF, 1 LF2, 2 LFMN2) on the current
        sigma, momenta and the kit's phi / inverted_phi."""
        self.lib.gnref_evolve_in_time(int(which), float(eps), int(steps))

    def condensate(self, tol=1e-9):
        out = np.zeros(11)
        self.lib.gnref_condensate(tol, _p(out))
        return out

    # ---- observables.c:323 and the lattice file (simulation.c:129-401) ----
    COUNTER_INTS = ("story_link", "story_sigma", "story_pi", "accepted_link", "done_link", "accepted_sigma",
                    "done_sigma", "accepted_pi", "done_pi", "measure")

    def condensate_sigma(self):
        """CondensateSigmaPi of the current sigma: the 8 outputs in its argument order."""
        out = np.zeros(8)
        self.lib.gnref_condensate_sigma(_p(out))
        return out

    def write_lattice(self, path, copy, counters):
        """WriteBinaryLattice of the current sigma (links: identity); counters a dict
        with epsilon_link, epsilon_pi and the COUNTER_INTS keys."""
        eps = np.array([counters["epsilon_link"], counters["epsilon_pi"]], dtype=np.float64)
        ints = (C.c_int * 10)(*[int(counters[k]) for k in self.COUNTER_INTS])
        self.lib.gnref_write_lattice(str(path).encode(), str(copy).encode(), _p(eps), ints)

    def read_lattice(self, path, copy):
        """ReadBinaryLattice(path, try_copy): returns (sigma, counters, check),
        check = TestWriteReadLattice of what was read.  Only for files that read
        in full (the reference exits otherwise)."""
        eps = np.zeros(2)
        ints = (C.c_int * 10)()
        check = self.lib.gnref_read_lattice(str(path).encode(), str(copy).encode(), _p(eps), ints)
        counters = {"epsilon_link": float(eps[0]), "epsilon_pi": float(eps[1])}
        counters.update({k: int(ints[i]) for i, k in enumerate(self.COUNTER_INTS)})
        return self.sigma(), counters, check

    # ---- the U(1) model (a build with extra_defs=("-DPI_INTERACTION",)) ----
    def _getv(self, name):
        v = np.empty(self.V)
        getattr(self.lib, name)(_p(v))
        return v

    def gauss2(self, npairs):
        """npairs Gauss2MeanVariance(.., 0, 1) pairs, as the pi momenta draw them: (npairs, 2)."""
        out = np.empty((npairs, 2))
        a, b = C.c_double(), C.c_double()
        for i in range(npairs):
            self.lib.gnref_gauss2(C.byref(a), C.byref(b))
            out[i] = (a.value, b.value)
        return out

    def set_pi(self, pi):
        self.lib.gnref_set_pi(_p(np.ascontiguousarray(pi, np.float64)))

    def pi(self):
        return self._getv("gnref_get_pi")

    def pimass(self):
        return self._getv("gnref_get_pimass")

    def set_pi_momenta(self, P):
        self.lib.gnref_set_pi_momenta(_p(np.ascontiguousarray(P, np.float64)))

    def pi_momenta(self):
        return self._getv("gnref_get_pi_momenta")

    def pi_force_buf(self):
        return self._getv("gnref_get_pi_force")

    def set_pi_params(self, eps, steps):
        self.lib.gnref_set_pi_params(eps, steps)

    def pi_force(self):
        return bool(self.lib.gnref_pi_force())

    def energy_pi(self):
        return self.lib.gnref_energy_pi()

    def trajectory_pi(self, accfile: str):
        """LeapFrog2Pi; returns (ok, accepted, dH parsed from the acceptance line)."""
        acc = C.c_int(0)
        ok = self.lib.gnref_trajectory_pi(accfile.encode(), C.byref(acc))
        dH = None
        if ok:
            with open(accfile) as fh:
                last = fh.read().strip().splitlines()[-1]
            dH = float(last.split("\t")[11])
        return bool(ok), bool(acc.value), dH
