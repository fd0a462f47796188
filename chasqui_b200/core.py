"""ctypes binding of the C ABI in include/chq.h (libchq.so, built in-tree by build.py).

There is no CPU fallback: if the CUDA library is missing or fails to load, every entry
point raises. Arrays cross the boundary as float64 numpy arrays in the reference's packed
layout (cells (ncomp, nk, nj, ni), faces/edges (ncomp, nk+1, nj+1, ni+1)).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .params import Params, config_from_params

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libchq.so")

FIELDS = ("u0", "u1", "w", "bcc", "ecc", "b1f0", "b2f0", "b3f0", "b1f1", "b2f1", "b3f1", "f1", "f2", "f3",
          "e2x1", "e3x1", "e1x2", "e3x2", "e1x3", "e2x3", "e1", "e2", "e3", "flag")
NCOMP = {"u0": 6, "u1": 6, "w": 6, "bcc": 3, "ecc": 3, "f1": 6, "f2": 6, "f3": 6}
CELL_FIELDS = {"u0", "u1", "w", "bcc", "ecc", "flag"}


class ChqError(RuntimeError):
    pass


class chq_config(C.Structure):
    _fields_ = [
        ("nx1", C.c_int), ("nx2", C.c_int), ("nx3", C.c_int), ("nghost", C.c_int),
        ("x1min", C.c_double), ("x1max", C.c_double), ("x2min", C.c_double), ("x2max", C.c_double),
        ("x3min", C.c_double), ("x3max", C.c_double),
        ("recon", C.c_int), ("rsolver", C.c_int), ("integrator", C.c_int),
        ("bc1", C.c_int), ("bc2", C.c_int), ("bc3", C.c_int),
        ("gamma", C.c_double), ("dfloor", C.c_double), ("pfloor", C.c_double), ("cfl", C.c_double),
        ("de_eta", C.c_double), ("lhlld_phi", C.c_double),
        ("dual_energy", C.c_int), ("low_mach", C.c_int), ("flatten", C.c_int), ("characteristic", C.c_int),
        ("fofc", C.c_int), ("flux_limiter", C.c_int),
        ("nu", C.c_double), ("kappa", C.c_double), ("eta", C.c_double), ("sts", C.c_int),
        ("precision", C.c_int), ("tlim", C.c_double), ("nlim", C.c_int),
        ("gravity_uniform", C.c_int), ("gravity_point", C.c_int),
        ("g1", C.c_double), ("g2", C.c_double), ("g3", C.c_double), ("gm", C.c_double),
        ("gx0", C.c_double), ("gy0", C.c_double), ("gz0", C.c_double), ("rsoft", C.c_double),
        ("cooling", C.c_int), ("lambda0", C.c_double), ("cool_alpha", C.c_double), ("tfloor", C.c_double),
    ]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
# (name, restype, argtypes) of every function declared in include/chq.h
SIGNATURES = [
    ("chq_config_defaults", None, [C.POINTER(chq_config)]),
    ("chq_mesh_create", C.c_int, [C.POINTER(chq_config), C.POINTER(_P)]),
    ("chq_mesh_destroy", C.c_int, [_P]),
    ("chq_mesh_dims", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("chq_mesh_bytes", C.c_longlong, [_P]),
    ("chq_config_bytes", C.c_longlong, [C.POINTER(chq_config)]),
    ("chq_init_problem", C.c_int, [_P, C.c_int, _D, C.c_int, _P]),
    ("chq_last_error", C.c_char_p, []),
    ("chq_array_size", C.c_long, [_P, C.c_char_p]),
    ("chq_upload", C.c_int, [_P, C.c_char_p, _D, C.c_long, _P]),
    ("chq_download", C.c_int, [_P, C.c_char_p, _D, C.c_long, _P]),
    ("chq_snapshot", C.c_int, [_P, C.c_int, C.POINTER(C.c_char_p), C.POINTER(_D), C.POINTER(C.c_long)]),
    ("chq_snapshot_wait", C.c_int, [_P]),
    ("chq_fluxes", C.c_int, [_P, C.c_int, C.c_int, _P]),
    ("chq_fluxes_all", C.c_int, [_P, C.c_int, _P]),
    ("chq_corner_emf", C.c_int, [_P, _P]),
    ("chq_update", C.c_int, [_P, C.c_int, C.c_double, C.c_double, C.c_double, _P]),
    ("chq_boundaries", C.c_int, [_P, C.c_int, _P]),
    ("chq_cons_to_prim", C.c_int, [_P, C.c_int, C.c_int, _D, _P]),
    ("chq_fofc_flag", C.c_int, [_P, C.c_int, C.POINTER(C.c_int), _P]),
    ("chq_fofc_repair", C.c_int, [_P, C.c_int, C.c_int, _P]),
    ("chq_limit_fluxes", C.c_int, [_P, C.c_int, C.c_double, C.POINTER(C.c_long), _P]),
    ("chq_stage", C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _P]),
    ("chq_prime", C.c_int, [_P, C.c_double, _P]),
    ("chq_cycles", C.c_int, [_P, C.c_int, _P]),
    ("chq_clock", C.c_int, [_P, _D, C.POINTER(C.c_int), _D, _D]),
    ("chq_counters", C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    ("chq_sts_stages", C.c_longlong, [_P]),
    ("chq_autotune", C.c_int, [_P, C.POINTER(C.c_int), _D]),
    ("chq_set_seglen", C.c_int, [_P, C.c_int]),
    ("chq_get_seglen", C.c_int, [_P]),
    ("chq_autotune2", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), _D, _D]),
    ("chq_set_xvariant", C.c_int, [_P, C.c_int]),
    ("chq_get_xvariant", C.c_int, [_P]),
    ("chq_set_yzvariant", C.c_int, [_P, C.c_int]),
    ("chq_get_yzvariant", C.c_int, [_P]),
    ("chq_autotune_yz", C.c_int, [_P, C.POINTER(C.c_int), _D]),
    ("chq_history", C.c_int, [_P, _D, _P]),
    ("chq_history_record", C.c_int, [_P, C.c_double, C.c_double, C.c_double, C.c_int]),
    ("chq_history_drain", C.c_int, [_P, _D, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), _D]),
    ("chq_run_host", C.c_int, [_P, _D, _D, _D, _D, C.c_int, C.c_double, _P]),
    ("chq_run_host_async", C.c_int, [_P, _D, _D, _D, _D, C.c_int, C.c_double]),
    ("chq_run_host_wait", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("chq_set_device", C.c_int, [C.c_int]),
    ("chq_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("chq_host_alloc", C.c_int, [C.c_longlong, C.POINTER(_P)]),
    ("chq_host_free", C.c_int, [_P]),
    ("chq_event_record", C.c_int, [_P, C.c_int]),
    ("chq_event_elapsed", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_float)]),
    ("chq_event_elapsed_between", C.c_int, [_P, C.c_int, _P, C.c_int, C.POINTER(C.c_float)]),
    ("chq_profile", C.c_int, [_P, C.c_int]),
    ("chq_profile_read", C.c_int, [_P, _D, C.POINTER(C.c_longlong), C.c_int]),
    ("chq_kernel_launches", C.c_longlong, [_P]),
    ("chq_batch_create", C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P)]),
    ("chq_batch_destroy", C.c_int, [_P]),
    ("chq_batch_cycles", C.c_int, [_P, C.c_int, _P]),
    ("chq_batch_set_graph", C.c_int, [_P, C.c_int]),
    ("chq_batch_status", C.c_int, [_P, _D, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("chq_batch_kernel_launches", C.c_longlong, [_P]),
    ("chq_batch_autotune", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), _D, _D]),
    ("chq_batch_stream", _P, [_P]),
    ("chq_server_create", C.c_int, [C.c_longlong, C.c_int, C.c_int, C.POINTER(_P)]),
    ("chq_server_submit", C.c_int, [_P, C.POINTER(chq_config), C.c_int, _D, C.c_int, C.POINTER(C.c_longlong)]),
    ("chq_server_step", C.c_int, [_P]),
    ("chq_server_status", C.c_int, [_P, C.c_longlong, C.c_void_p]),
    ("chq_server_job_mesh", _P, [_P, C.c_longlong]),
    ("chq_server_stats", C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_longlong), _D]),
    ("chq_server_destroy", C.c_int, [_P]),
    ("chq_server_set_lanes", C.c_int, [_P, C.c_int]),
    ("chq_server_set_solo_cells", C.c_int, [_P, C.c_longlong]),
    ("chq_server_set_solo_slots", C.c_int, [_P, C.c_int]),
    ("chq_server_set_autotune", C.c_int, [_P, C.c_int]),
    ("chq_history_noalloc", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      _P, _P, _P, _P, _D, _P]),
    ("chq_slab_create", C.c_int, [C.POINTER(chq_config), C.c_int, C.c_int, C.POINTER(_P)]),
    ("chq_slab_info", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("chq_slab_halo_bytes", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_longlong)]),
    ("chq_slab_pack", C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P, _P]),
    ("chq_slab_unpack", C.c_int, [_P, C.c_int, C.c_int, C.c_int, _P, _P]),
    ("chq_slab_ctl", C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    ("chq_slab_prime", C.c_int, [_P, C.c_double, C.c_int, _P]),
    ("chq_slab_begin", C.c_int, [_P, _P]),
    ("chq_slab_stage", C.c_int, [_P, C.c_int, C.c_int, _P]),
    ("chq_slab_end", C.c_int, [_P, _P]),
]

TUNE_LENGTHS = (4, 8, 16, 32, 64)   # CHQ_TUNE_LENGTHS
TUNE_NLEN = len(TUNE_LENGTHS)
TUNE_NXVAR = 2                       # CHQ_TUNE_NXVAR

PROFILE_KINDS = ("fluxes", "corner_emf", "update", "fofc_flag", "fofc_repair", "boundaries", "c2p_dt", "limiter",
                 "step_ctl", "diffusion", "sts")

_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load libchq.so once; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ChqError(f"CUDA library not built: {p} (run __graft_entry__.build() or make -C chasqui_b200/csrc)")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _check(rc: int) -> int:
    if rc < 0:
        msg = load_library().chq_last_error().decode(errors="replace")
        raise ChqError(f"chq error {rc}: {msg}")
    return rc


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


def default_config() -> chq_config:
    c = chq_config()
    load_library().chq_config_defaults(C.byref(c))
    return c


def make_config(**kw) -> chq_config:
    c = default_config()
    for k, v in kw.items():
        if not hasattr(c, k):
            raise ChqError(f"unknown config field {k}")
        setattr(c, k, v)
    return c


class Mesh:
    """A device mesh (one simulation) behind the C ABI."""

    def __init__(self, cfg: chq_config | None = None, **kw):
        lib = load_library()
        self.cfg = cfg if cfg is not None else make_config(**kw)
        h = _P()
        _check(self._create(lib, h))
        self._h = h
        d = (C.c_int * 10)()
        _check(lib.chq_mesh_dims(h, d))
        (self.nx1, self.nx2, self.nx3, self.ng, self.ni, self.nj, self.nk, self.nstage,
         two, three) = list(d)
        self.two_d, self.three_d = bool(two), bool(three)

    def _create(self, lib, h) -> int:
        return lib.chq_mesh_create(C.byref(self.cfg), C.byref(h))

    @classmethod
    def from_params(cls, pin: Params, **extra) -> "Mesh":
        c = config_from_params(pin)
        c.update(extra)
        return cls(make_config(**c))

    def close(self):
        if getattr(self, "_h", None):
            load_library().chq_mesh_destroy(self._h)   # waits for queued work, host jobs included
            self._h = None
        self._host_jobs = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- geometry ----
    @property
    def nbytes(self) -> int:
        return int(load_library().chq_mesh_bytes(self._h))

    def shape(self, name: str) -> tuple:
        if name == "vtk":   # the VTK dump's cell data: 8 big-endian float32 per cell, in doubles
            return (int(load_library().chq_array_size(self._h, b"vtk")),)
        nc = NCOMP.get(name, 1)
        if name in CELL_FIELDS:
            return (nc, self.nk, self.nj, self.ni)
        return (nc, self.nk + 1, self.nj + 1, self.ni + 1)

    # ---- transfer ----
    def snapshot(self, names) -> dict:
        """Start a non-stalling output snapshot of `names` (chq_snapshot) into new page-locked
        host arrays and return them; they are valid after snapshot_wait()."""
        pins = {n: PinnedArray(self.shape(n)) for n in names}
        keys = (C.c_char_p * len(names))(*[n.encode() for n in names])
        ptrs = (_D * len(names))(*[_dptr(pins[n].array) for n in names])
        sizes = (C.c_long * len(names))(*[pins[n].array.size for n in names])
        _check(load_library().chq_snapshot(self._h, len(names), keys, ptrs, sizes))
        self._snap = pins   # keep the buffers alive while the copy is in flight
        return pins

    def snapshot_wait(self) -> dict:
        """Wait for the snapshot and return its fields as ordinary numpy arrays (copied out of
        the page-locked buffers, which are released here)."""
        _check(load_library().chq_snapshot_wait(self._h))
        pins = getattr(self, "_snap", {})
        self._snap = {}
        out = {}
        for n, p in pins.items():
            a = np.array(p.array, copy=True)
            out[n] = a if a.shape[0] > 1 else a[0]
        return out

    def get(self, name: str) -> np.ndarray:
        shp = self.shape(name)
        out = np.empty(shp, dtype=np.float64)
        _check(load_library().chq_download(self._h, name.encode(), _dptr(out), out.size, None))
        return out if shp[0] > 1 else out[0]

    def set(self, name: str, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        n = load_library().chq_array_size(self._h, name.encode())
        if a.size != n:
            raise ChqError(f"{name}: expected {n} values, got {a.size}")
        _check(load_library().chq_upload(self._h, name.encode(), _dptr(a), a.size, None))

    def init_problem(self, problem: str, params) -> None:
        """Device problem generator: 'orszag_tang' {beta}, 'cpaw' {m1,m2,m3,dens,pres,b_par,amp},
        'blast' {pres_in,pres_out,radius,b0,angle_deg,noise_amp,seed}. Call prime() next."""
        pid = {"orszag_tang": 0, "cpaw": 1, "blast": 2}[problem]
        a = np.ascontiguousarray(params, dtype=np.float64)
        _check(load_library().chq_init_problem(self._h, pid, _dptr(a), a.size, None))

    # ---- stage seam ----
    def fluxes(self, dir: int, cur: int = 0):
        _check(load_library().chq_fluxes(self._h, dir, cur, None))

    def fluxes_all(self, cur: int = 0):
        _check(load_library().chq_fluxes_all(self._h, cur, None))

    def corner_emf(self):
        _check(load_library().chq_corner_emf(self._h, None))

    def update(self, out: int, g0: float, g1: float, beta_dt: float):
        _check(load_library().chq_update(self._h, out, g0, g1, beta_dt, None))

    def boundaries(self, buf: int = 0):
        _check(load_library().chq_boundaries(self._h, buf, None))

    def cons_to_prim(self, buf: int = 0, compute_dt: bool = True) -> float | None:
        v = C.c_double(0.0)
        _check(load_library().chq_cons_to_prim(self._h, buf, int(compute_dt), C.byref(v) if compute_dt else None, None))
        return v.value if compute_dt else None

    def fofc_flag(self, buf: int) -> int:
        n = C.c_int(0)
        _check(load_library().chq_fofc_flag(self._h, buf, C.byref(n), None))
        return n.value

    def fofc_repair(self, dir: int, cur: int):
        _check(load_library().chq_fofc_repair(self._h, dir, cur, None))

    def limit_fluxes(self, dir: int, beta_dt: float) -> int:
        n = C.c_long(0)
        _check(load_library().chq_limit_fluxes(self._h, dir, beta_dt, C.byref(n), None))
        return n.value

    def stage(self, cur: int, out: int, g0: float, g1: float, beta_dt: float):
        _check(load_library().chq_stage(self._h, cur, out, g0, g1, beta_dt, None))

    # ---- cycles ----
    def prime(self, t: float = 0.0):
        _check(load_library().chq_prime(self._h, t, None))

    def cycles(self, n: int):
        _check(load_library().chq_cycles(self._h, n, None))

    def clock(self) -> dict:
        t, dt, mdt = C.c_double(), C.c_double(), C.c_double()
        cyc = C.c_int()
        _check(load_library().chq_clock(self._h, C.byref(t), C.byref(cyc), C.byref(dt), C.byref(mdt)))
        return {"t": t.value, "cycle": cyc.value, "dt": dt.value, "min_dt": mdt.value}

    def counters(self) -> tuple[int, int]:
        a, b = C.c_longlong(), C.c_longlong()
        _check(load_library().chq_counters(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def sts_stages(self) -> int:
        return int(load_library().chq_sts_stages(self._h))

    def autotune(self) -> dict:
        """Pick the y/z march length and the x-sweep variant of the flux kernel by timing it on
        this mesh's state (call after prime). Returns {"seglen": best length, "ms": {length: ms
        per launch}, "xvar": best variant, "xvar_ms": {variant: ms per launch}}."""
        best, bx = C.c_int(), C.c_int()
        ms, msx = np.zeros(TUNE_NLEN), np.zeros(TUNE_NXVAR)
        _check(load_library().chq_autotune2(self._h, C.byref(best), C.byref(bx), _dptr(ms), _dptr(msx)))
        return {"seglen": best.value, "ms": {L: float(t) for L, t in zip(TUNE_LENGTHS, ms)},
                "xvar": bx.value, "xvar_ms": {v: float(t) for v, t in enumerate(msx)}}

    @property
    def xvariant(self) -> int:
        return int(load_library().chq_get_xvariant(self._h))

    @xvariant.setter
    def xvariant(self, v: int) -> None:
        _check(load_library().chq_set_xvariant(self._h, int(v)))

    @property
    def yzvariant(self) -> int:
        return int(load_library().chq_get_yzvariant(self._h))

    @yzvariant.setter
    def yzvariant(self, v: int) -> None:
        _check(load_library().chq_set_yzvariant(self._h, int(v)))

    def autotune_yz(self) -> dict:
        """Time the y/z staging variants (cp.async, TMA) of the FP64 streaming-PPM flux launch
        on this mesh's state and keep the faster: {"yzvar": chosen, "ms": {0: ms, 1: ms}}."""
        v = C.c_int()
        ms = np.zeros(2)
        _check(load_library().chq_autotune_yz(self._h, C.byref(v), _dptr(ms)))
        return {"yzvar": v.value, "ms": {0: float(ms[0]), 1: float(ms[1])}}

    @property
    def seglen(self) -> int:
        return int(load_library().chq_get_seglen(self._h))

    @seglen.setter
    def seglen(self, n: int) -> None:
        _check(load_library().chq_set_seglen(self._h, int(n)))

    def history(self) -> np.ndarray:
        out = np.zeros(10)
        _check(load_library().chq_history(self._h, _dptr(out), None))
        return out

    def record_history(self, dt_hst: float, next_t: float, eps: float = 0.0, capacity: int = 256) -> None:
        """Record .hst rows on the device at the end of each cycle reaching the next output time
        (capacity 0: off)."""
        _check(load_library().chq_history_record(self._h, float(dt_hst), float(next_t), float(eps), int(capacity)))

    def drain_history(self, max_rows: int = 256):
        """(rows (n x 12: t, dt, the ten history values), rows lost, next output time)."""
        rows = np.zeros((max(int(max_rows), 1), 12))
        n, lost, nxt = C.c_int(), C.c_int(), np.zeros(1)
        _check(load_library().chq_history_drain(self._h, _dptr(rows), int(max_rows), C.byref(n), C.byref(lost),
                                                _dptr(nxt)))
        return rows[:n.value].copy(), lost.value, float(nxt[0])

    def run_host(self, u: np.ndarray, b1: np.ndarray, b2: np.ndarray, b3: np.ndarray, ncycles: int,
                 t0: float = 0.0) -> int:
        for a in (u, b1, b2, b3):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ChqError("run_host needs C-contiguous float64 arrays")
        return _check(load_library().chq_run_host(self._h, _dptr(u), _dptr(b1), _dptr(b2), _dptr(b3), ncycles, t0, None))

    def run_host_async(self, u: np.ndarray, b1: np.ndarray, b2: np.ndarray, b3: np.ndarray, ncycles: int,
                       t0: float = 0.0):
        """Queue run_host's job without waiting (up to two per mesh); the arrays must be
        page-locked (PinnedArray) and are held until the run_host_wait() that returns it."""
        for a in (u, b1, b2, b3):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ChqError("run_host_async needs C-contiguous float64 arrays")
        _check(load_library().chq_run_host_async(self._h, _dptr(u), _dptr(b1), _dptr(b2), _dptr(b3), ncycles, t0))
        if getattr(self, "_host_jobs", None) is None:
            self._host_jobs = []
        self._host_jobs.append((u, b1, b2, b3))

    def run_host_wait(self) -> int:
        """Wait for the oldest queued host job; its cycle count."""
        c = C.c_int()
        _check(load_library().chq_run_host_wait(self._h, C.byref(c)))
        self._host_jobs.pop(0)
        return int(c.value)

    # ---- timing ----
    def record(self, slot: int):
        _check(load_library().chq_event_record(self._h, slot))

    def elapsed_ms(self, a: int, b: int) -> float:
        v = C.c_float()
        _check(load_library().chq_event_elapsed(self._h, a, b, C.byref(v)))
        return float(v.value)

    def elapsed_ms_to(self, a: int, other: "Mesh", b: int) -> float:
        """device time from this mesh's slot a to the other mesh's slot b"""
        v = C.c_float()
        _check(load_library().chq_event_elapsed_between(self._h, a, other._h, b, C.byref(v)))
        return float(v.value)

    def kernel_launches(self) -> int:
        return int(load_library().chq_kernel_launches(self._h))

    def profile(self, on: bool = True):
        _check(load_library().chq_profile(self._h, int(on)))

    def profile_read(self, reset: bool = True) -> dict:
        ms = (C.c_double * len(PROFILE_KINDS))()
        n = (C.c_longlong * len(PROFILE_KINDS))()
        _check(load_library().chq_profile_read(self._h, ms, n, int(reset)))
        return {k: (ms[q], n[q]) for q, k in enumerate(PROFILE_KINDS)}

    def set_state(self, u0, b1, b2, b3):
        self.set("u0", u0)
        self.set("b1f0", b1)
        self.set("b2f0", b2)
        self.set("b3f0", b3)


class chq_job_status(C.Structure):
    _fields_ = [("state", C.c_int), ("cycle", C.c_int), ("t", C.c_double), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double), ("zone_updates", C.c_longlong),
                ("bytes", C.c_longlong), ("history", C.c_double * 10)]


JOB_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}
PGEN = {"orszag_tang": 0, "cpaw": 1, "blast": 2}


class Server:
    """Continuous-batching simulation server (chq_server_*)."""

    def __init__(self, hbm_budget_bytes: int, max_active: int = 1024, cycles_per_step: int = 4, lanes: int = 8,
                 solo_cells: int = None, autotune: bool = False, solo_slots: int = None):
        h = _P()
        _check(load_library().chq_server_create(int(hbm_budget_bytes), max_active, cycles_per_step, C.byref(h)))
        _check(load_library().chq_server_set_autotune(h, int(bool(autotune))))
        self._h = h
        _check(load_library().chq_server_set_lanes(h, int(lanes)))
        if solo_cells is not None:
            _check(load_library().chq_server_set_solo_cells(h, int(solo_cells)))
        if solo_slots is not None:
            _check(load_library().chq_server_set_solo_slots(h, int(solo_slots)))

    def submit(self, cfg: chq_config, problem: str, params) -> int:
        a = np.ascontiguousarray(params, dtype=np.float64)
        jid = C.c_longlong()
        _check(load_library().chq_server_submit(self._h, C.byref(cfg), PGEN[problem], _dptr(a), a.size, C.byref(jid)))
        return jid.value

    def step(self) -> int:
        return _check(load_library().chq_server_step(self._h))

    def status(self, jid: int) -> dict:
        st = chq_job_status()
        _check(load_library().chq_server_status(self._h, jid, C.byref(st)))
        return {"state": JOB_STATES[st.state], "cycle": st.cycle, "t": st.t, "t_submit": st.t_submit,
                "t_start": st.t_start, "t_done": st.t_done, "zone_updates": st.zone_updates, "bytes": st.bytes,
                "history": list(st.history)}

    def job_mesh_handle(self, jid: int):
        return load_library().chq_server_job_mesh(self._h, jid)

    def stats(self) -> dict:
        used, za = C.c_longlong(), C.c_longlong()
        act, q = C.c_int(), C.c_int()
        clk = C.c_double()
        _check(load_library().chq_server_stats(self._h, C.byref(used), C.byref(act), C.byref(q), C.byref(za),
                                               C.byref(clk)))
        return {"used_bytes": used.value, "active": act.value, "queued": q.value, "zone_updates": za.value,
                "clock": clk.value}

    def close(self):
        if getattr(self, "_h", None):
            load_library().chq_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many primed meshes of one class stepped together, one launch per kernel kind per stage."""

    def __init__(self, meshes, graph: bool = False):
        lib = load_library()
        self.meshes = list(meshes)
        arr = (_P * len(self.meshes))(*[m._h for m in self.meshes])
        h = _P()
        _check(lib.chq_batch_create(arr, len(self.meshes), C.byref(h)))
        self._h = h
        if graph:
            _check(lib.chq_batch_set_graph(h, 1))

    def cycles(self, n: int):
        _check(load_library().chq_batch_cycles(self._h, n, None))

    def status(self):
        n = len(self.meshes)
        t = (C.c_double * n)()
        cyc = (C.c_int * n)()
        done = (C.c_int * n)()
        _check(load_library().chq_batch_status(self._h, t, cyc, done))
        return [{"t": t[j], "cycle": cyc[j], "done": bool(done[j])} for j in range(n)]

    def kernel_launches(self) -> int:
        return int(load_library().chq_batch_kernel_launches(self._h))

    def autotune(self) -> dict:
        """The batch's march length and x-sweep variant, timed on the batched flux launch over
        all members (cached per scheme, precision and size class)."""
        best, bx = C.c_int(), C.c_int()
        ms, msx = np.zeros(TUNE_NLEN), np.zeros(TUNE_NXVAR)
        _check(load_library().chq_batch_autotune(self._h, C.byref(best), C.byref(bx), _dptr(ms), _dptr(msx)))
        return {"seglen": best.value, "ms": {L: float(t) for L, t in zip(TUNE_LENGTHS, ms)},
                "xvar": bx.value, "xvar_ms": {v: float(t) for v, t in enumerate(msx)}}

    def close(self):
        if getattr(self, "_h", None):
            load_library().chq_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_device(dev: int) -> None:
    _check(load_library().chq_set_device(dev))


def device_count() -> int:
    n = C.c_int(0)
    _check(load_library().chq_device_count(C.byref(n)))
    return n.value


class PinnedArray:
    """A float64 numpy array in page-locked host memory (freed with the object)."""

    def __init__(self, shape):
        n = int(np.prod(shape))
        p = _P()
        _check(load_library().chq_host_alloc(8 * max(n, 1), C.byref(p)))
        self._p = p
        buf = (C.c_double * max(n, 1)).from_address(p.value)
        buf._owner = self   # numpy views keep the buffer, the buffer keeps the allocation
        self.array = np.frombuffer(buf, dtype=np.float64, count=n).reshape(shape)

    def __del__(self):
        try:
            if self._p:
                load_library().chq_host_free(self._p)
                self._p = None
        except Exception:
            pass
