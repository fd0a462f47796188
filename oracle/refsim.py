"""ctypes binding of oracle/_ref/libchqref.so: the reference's own kernels compiled in place
against the project's Kokkos-API shim (see oracle/Makefile and oracle/ref_capi.cpp).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libchqref.so")

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_SIGS = [
    ("chqref_last_error", C.c_char_p, []),
    ("chqref_set_threads", None, [C.c_int]),
    ("chqref_get_threads", C.c_int, []),
    ("chqref_open", _P, [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), C.c_char_p]),
    ("chqref_close", None, [_P]),
    ("chqref_dims", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("chqref_time", C.c_double, [_P]),
    ("chqref_cycle", C.c_int, [_P]),
    ("chqref_min_dt", C.c_double, [_P]),
    ("chqref_fofc_count", C.c_long, [_P]),
    ("chqref_limiter_count", C.c_long, [_P]),
    ("chqref_sts_stages", C.c_long, [_P]),
    ("chqref_set_time", None, [_P, C.c_double, C.c_double]),
    ("chqref_array_size", C.c_long, [_P, C.c_char_p]),
    ("chqref_get", C.c_int, [_P, C.c_char_p, _D, C.c_long]),
    ("chqref_set", C.c_int, [_P, C.c_char_p, _D, C.c_long]),
    ("chqref_prime", C.c_int, [_P]),
    ("chqref_cycles", C.c_int, [_P, C.c_int]),
    ("chqref_stage", C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]),
    ("chqref_cons_to_prim", C.c_double, [_P, C.c_int, C.c_int]),
    ("chqref_boundaries", C.c_int, [_P, C.c_int]),
    ("chqref_fluxes", C.c_int, [_P, C.c_int, C.c_int]),
    ("chqref_corner_emf", C.c_int, [_P]),
    ("chqref_update", C.c_int, [_P, C.c_int, C.c_double, C.c_double, C.c_double]),
    ("chqref_fofc_flag", C.c_int, [_P, C.c_int]),
    ("chqref_fofc_repair", C.c_int, [_P, C.c_int, C.c_int]),
    ("chqref_limit_fluxes", C.c_long, [_P, C.c_int, C.c_double]),
    ("chqref_history", C.c_int, [_P, _D]),
    ("chqref_write_vtk", C.c_int, [_P, C.c_char_p]),
    ("chqref_write_restart", C.c_int, [_P, C.c_char_p]),
    ("chqref_recon", C.c_int, [C.c_int, _D, C.c_long, _D, _D]),
    ("chqref_flattening", C.c_int, [_D, _D, _D, C.c_long, _D]),
    ("chqref_riemann", C.c_int, [C.c_int, _D, _D, _D, C.c_long, C.c_double, _D, _D, _D]),
    ("chqref_eigen", C.c_int, [_D, C.c_long, C.c_double, _D, _D]),
]

_lib = None


def available() -> bool:
    return os.path.exists(REF_LIB)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference oracle not built: {REF_LIB} (make -C oracle REF=<reference source tree>)")
        _lib = C.CDLL(REF_LIB)
        for n, r, a in _SIGS:
            f = getattr(_lib, n)
            f.restype = r
            f.argtypes = a
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_D)


CELL = {"u0", "u1", "w", "bcc", "ecc", "flag"}
NCOMP = {"u0": 6, "u1": 6, "w": 6, "bcc": 3, "ecc": 3, "f1": 6, "f2": 6, "f3": 6}


class RefSim:
    """One reference simulation (Mesh + Physics + clock) driven kernel by kernel."""

    def __init__(self, params_text: str, overrides=(), restart: str | None = None, threads: int | None = None):
        L = lib()
        if threads:
            L.chqref_set_threads(int(threads))
        fd, self._infile = tempfile.mkstemp(suffix=".in", prefix="chqref_")
        with os.fdopen(fd, "w") as f:
            f.write(params_text)
        ov = [o.encode() for o in overrides]
        arr = (C.c_char_p * max(1, len(ov)))(*ov)
        self._h = L.chqref_open(self._infile.encode(), len(ov), arr, (restart or "").encode())
        if not self._h:
            raise RuntimeError("reference open failed: " + L.chqref_last_error().decode())
        d = (C.c_int * 10)()
        L.chqref_dims(self._h, d)
        (self.nx1, self.nx2, self.nx3, self.ng, self.ni, self.nj, self.nk, self.nstage, two, three) = list(d)
        self.two_d, self.three_d = bool(two), bool(three)

    def close(self):
        if getattr(self, "_h", None):
            lib().chqref_close(self._h)
            self._h = None
            try:
                os.unlink(self._infile)
            except OSError:
                pass

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, name):
        nc = NCOMP.get(name, 1)
        if name in CELL:
            return (nc, self.nk, self.nj, self.ni)
        return (nc, self.nk + 1, self.nj + 1, self.ni + 1)

    def get(self, name):
        shp = self.shape(name)
        out = np.empty(shp)
        if lib().chqref_get(self._h, name.encode(), _d(out), out.size) != 0:
            raise RuntimeError("bad field " + name)
        return out if shp[0] > 1 else out[0]

    def set(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if lib().chqref_set(self._h, name.encode(), _d(a), a.size) != 0:
            raise RuntimeError("bad field " + name)

    # pass-throughs
    def prime(self):
        lib().chqref_prime(self._h)

    def cycles(self, n):
        return lib().chqref_cycles(self._h, n)

    def stage(self, cur, out, g0, g1, bdt):
        lib().chqref_stage(self._h, cur, out, g0, g1, bdt)

    def cons_to_prim(self, buf=0, compute_dt=True):
        return lib().chqref_cons_to_prim(self._h, buf, int(compute_dt))

    def boundaries(self, buf=0):
        lib().chqref_boundaries(self._h, buf)

    def fluxes(self, d, cur=0):
        lib().chqref_fluxes(self._h, d, cur)

    def corner_emf(self):
        lib().chqref_corner_emf(self._h)

    def update(self, out, g0, g1, bdt):
        lib().chqref_update(self._h, out, g0, g1, bdt)

    def fofc_flag(self, buf):
        return lib().chqref_fofc_flag(self._h, buf)

    def fofc_repair(self, d, cur):
        lib().chqref_fofc_repair(self._h, d, cur)

    def limit_fluxes(self, d, bdt):
        return lib().chqref_limit_fluxes(self._h, d, bdt)

    def history(self):
        out = np.zeros(10)
        lib().chqref_history(self._h, _d(out))
        return out

    @property
    def time(self):
        return lib().chqref_time(self._h)

    @property
    def cycle(self):
        return lib().chqref_cycle(self._h)

    @property
    def min_dt(self):
        return lib().chqref_min_dt(self._h)

    @property
    def fofc_count(self):
        return lib().chqref_fofc_count(self._h)

    @property
    def sts_stages(self):
        return lib().chqref_sts_stages(self._h)

    def set_time(self, t, tlim):
        lib().chqref_set_time(self._h, t, tlim)

    def write_vtk(self, fname):
        return lib().chqref_write_vtk(self._h, fname.encode())

    def write_restart(self, fname):
        return lib().chqref_write_restart(self._h, fname.encode())


# ---- point functions of the reference (src/recon.hpp, src/riemann.hpp, src/eigen_mhd.hpp) ----
def recon(scheme: int, q: np.ndarray):
    q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, 6)
    n = q.shape[0]
    ql, qr = np.empty(n), np.empty(n)
    lib().chqref_recon(scheme, _d(q), n, _d(ql), _d(qr))
    return ql, qr


def flattening(p5, um1, up1):
    p5 = np.ascontiguousarray(p5, dtype=np.float64).reshape(-1, 5)
    um1 = np.ascontiguousarray(um1, dtype=np.float64)
    up1 = np.ascontiguousarray(up1, dtype=np.float64)
    out = np.empty(p5.shape[0])
    lib().chqref_flattening(_d(p5), _d(um1), _d(up1), p5.shape[0], _d(out))
    return out


def riemann(solver: int, L, R, bn, gamma, theta=None, phi=None):
    L = np.ascontiguousarray(L, dtype=np.float64).reshape(-1, 7)
    R = np.ascontiguousarray(R, dtype=np.float64).reshape(-1, 7)
    bn = np.ascontiguousarray(bn, dtype=np.float64)
    n = L.shape[0]
    th = np.ascontiguousarray(theta if theta is not None else np.ones(n), dtype=np.float64)
    ph = np.ascontiguousarray(phi if phi is not None else np.ones(n), dtype=np.float64)
    f = np.empty((n, 7))
    lib().chqref_riemann(solver, _d(L), _d(R), _d(bn), n, gamma, _d(th), _d(ph), _d(f))
    return f


def eigen(w8, gamma):
    w8 = np.ascontiguousarray(w8, dtype=np.float64).reshape(-1, 8)
    n = w8.shape[0]
    Lm, Rm = np.empty((n, 7, 7)), np.empty((n, 7, 7))
    lib().chqref_eigen(_d(w8), n, gamma, _d(Lm), _d(Rm))
    return Lm, Rm
