"""ctypes binding of oracle/_port/libchqport.so, the plain-C restatement of the path.

Test infrastructure only (tests/, smoke, bench's CPU baseline)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_port", "libchqport.so")


class port_cfg(C.Structure):
    _fields_ = [("nx1", C.c_int), ("nx2", C.c_int), ("nx3", C.c_int), ("ng", C.c_int),
                ("x1min", C.c_double), ("x1max", C.c_double), ("x2min", C.c_double), ("x2max", C.c_double),
                ("x3min", C.c_double), ("x3max", C.c_double),
                ("recon", C.c_int), ("rsolver", C.c_int), ("nstage", C.c_int), ("bc", C.c_int * 3),
                ("gamma", C.c_double), ("dfloor", C.c_double), ("pfloor", C.c_double), ("cfl", C.c_double),
                ("de_eta", C.c_double), ("lhlld_phi", C.c_double), ("tlim", C.c_double),
                ("dual_energy", C.c_int), ("low_mach", C.c_int), ("flatten", C.c_int), ("characteristic", C.c_int),
                ("fofc", C.c_int), ("flux_limiter", C.c_int),
                ("nu", C.c_double), ("kappa", C.c_double), ("eta", C.c_double), ("sts", C.c_int),
                ("grav_uniform", C.c_int), ("grav_point", C.c_int), ("g1", C.c_double), ("g2", C.c_double),
                ("g3", C.c_double), ("gm", C.c_double), ("gx0", C.c_double), ("gy0", C.c_double),
                ("gz0", C.c_double), ("rsoft", C.c_double), ("cooling", C.c_int), ("lambda0", C.c_double),
                ("cool_alpha", C.c_double), ("tfloor", C.c_double)]


_P, _D = C.c_void_p, C.POINTER(C.c_double)
_SIGS = [("port_create", _P, [C.POINTER(port_cfg)]), ("port_destroy", None, [_P]),
         ("port_size", C.c_long, [_P, C.c_char_p]), ("port_get", C.c_int, [_P, C.c_char_p, _D, C.c_long]),
         ("port_set", C.c_int, [_P, C.c_char_p, _D, C.c_long]), ("port_fluxes", None, [_P, C.c_int, C.c_int]),
         ("port_corner_emf", None, [_P]), ("port_update", None, [_P, C.c_int, C.c_double, C.c_double, C.c_double]),
         ("port_boundaries", None, [_P, C.c_int]), ("port_cons_to_prim", C.c_double, [_P, C.c_int, C.c_int]),
         ("port_fofc_flag", C.c_int, [_P, C.c_int]), ("port_fofc_repair", None, [_P, C.c_int, C.c_int]),
         ("port_limit_fluxes", C.c_long, [_P, C.c_int, C.c_double]),
         ("port_stage", None, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]),
         ("port_prime", None, [_P, C.c_double]), ("port_cycles", C.c_int, [_P, C.c_int]),
         ("port_clock", None, [_P, _D, C.POINTER(C.c_int), _D, C.POINTER(C.c_long)]),
         ("port_history", None, [_P, _D]), ("port_set_threads", None, [C.c_int]),
         ("port_sts_stages", C.c_long, [_P]),
         ("port_recon", None, [C.c_int, _D, _D, _D]),
         ("port_riemann", None, [C.c_int, _D, _D, C.c_double, C.c_double, C.c_double, C.c_double, _D])]
_lib = None


def available() -> bool:
    return os.path.exists(PORT_LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"oracle port not built: {PORT_LIB} (make -C oracle)")
        _lib = C.CDLL(PORT_LIB)
        for n, r, a in _SIGS:
            f = getattr(_lib, n)
            f.restype, f.argtypes = r, a
    return _lib


def cfg_from_chq(c: dict) -> port_cfg:
    """port_cfg from the chq_config field dict of chasqui_b200.params.config_from_params."""
    p = port_cfg()
    for k in ("nx1", "nx2", "nx3", "x1min", "x1max", "x2min", "x2max", "x3min", "x3max", "recon", "rsolver", "gamma",
              "dfloor", "pfloor", "cfl", "de_eta", "lhlld_phi", "tlim", "dual_energy", "low_mach", "flatten",
              "characteristic", "fofc", "flux_limiter"):
        setattr(p, k, c[k])
    for k in ("nu", "kappa", "eta", "sts", "g1", "g2", "g3", "gm", "gx0", "gy0", "gz0", "rsoft", "cooling",
              "lambda0", "cool_alpha", "tfloor"):
        if k in c:
            setattr(p, k, c[k])
    p.grav_uniform = c.get("gravity_uniform", 0)
    p.grav_point = c.get("gravity_point", 0)
    if "cool_alpha" not in c:
        p.cool_alpha = 1.0
    p.ng = c["nghost"]
    p.nstage = c["integrator"]
    p.bc[0], p.bc[1], p.bc[2] = c["bc1"], c["bc2"], c["bc3"]
    return p


class PortSim:
    def __init__(self, cfg: port_cfg):
        self._h = lib().port_create(C.byref(cfg))
        self.cfg = cfg
        ng = cfg.ng
        self.ni = cfg.nx1 + 2 * ng
        self.nj = cfg.nx2 + 2 * ng if cfg.nx2 > 1 else 1
        self.nk = cfg.nx3 + 2 * ng if cfg.nx3 > 1 else 1

    def close(self):
        if self._h:
            lib().port_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get(self, name):
        n = lib().port_size(self._h, name.encode())
        out = np.empty(n)
        lib().port_get(self._h, name.encode(), out.ctypes.data_as(_D), n)
        return out

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        if lib().port_set(self._h, name.encode(), a.ctypes.data_as(_D), a.size) != 0:
            raise RuntimeError("bad field " + name)

    def prime(self, t=0.0):
        lib().port_prime(self._h, t)

    def cycles(self, n):
        return lib().port_cycles(self._h, n)

    def stage(self, cur, out, g0, g1, bdt):
        lib().port_stage(self._h, cur, out, g0, g1, bdt)

    def clock(self):
        t, mdt = C.c_double(), C.c_double()
        cyc, nf = C.c_int(), C.c_long()
        lib().port_clock(self._h, C.byref(t), C.byref(cyc), C.byref(mdt), C.byref(nf))
        return {"t": t.value, "cycle": cyc.value, "min_dt": mdt.value, "fofc": nf.value}

    def sts_stages(self):
        return lib().port_sts_stages(self._h)

    def history(self):
        out = np.zeros(10)
        lib().port_history(self._h, out.ctypes.data_as(_D))
        return out
