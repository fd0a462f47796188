"""The allocation-free history entry point (chq_history_noalloc) against chq_history.

It exists for callers that cannot allocate device memory (their own pool or framework owns
it, or they must avoid cudaMalloc's implicit synchronisation), so here the caller's state
lives in device buffers that the test allocates itself and fills with a mesh's state in the
reference layout. Two calls in a row must each match chq_history() on the same state to the
tolerance of the other history test (1e-12 relative). The file sorts last so that a run
stopping at the first failure has run every other test first; it also passes alone."""
import ctypes as C

import numpy as np
import pytest

from tests import cases
from tests.parity import copy_state, make_pair

pytestmark = pytest.mark.gpu


def _cudart():
    rt = C.CDLL("libcudart.so.12")
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaFree.argtypes = [C.c_void_p]
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return rt


class DeviceArrays:
    """Caller-owned device copies of host arrays (allocated by the caller, not the library)."""

    def __init__(self, *arrays):
        self.rt = _cudart()
        self.ptrs = []
        for a in arrays:
            a = np.ascontiguousarray(a, dtype=np.float64)
            p = C.c_void_p()
            assert self.rt.cudaMalloc(C.byref(p), a.nbytes) == 0
            assert self.rt.cudaMemcpy(p, a.ctypes.data, a.nbytes, 1) == 0
            self.ptrs.append(p)

    def free(self):
        for p in self.ptrs:
            self.rt.cudaFree(p)
        self.ptrs = []


# the 8 x 200 Orszag-Tang mesh splits its rows into two 128-row slabs, the second one clipped
# at the mesh edge; the shock tube is one-dimensional (one slab of one row)
@pytest.mark.parametrize("text,cycles", [(cases.blast(16), 3), (cases.ot(32), 4),
                                         (cases.ORSZAG_TANG.format(n=8).replace("nx2 = 8", "nx2 = 200"), 3),
                                         (cases.shock_tube(64), 5)],
                         ids=["blast3d", "ot2d", "ot2d_8x200", "shock1d"])
def test_noalloc_history_matches_history_twice(text, cycles):
    from chasqui_b200 import load_library
    ref, mesh = make_pair(text, [])
    copy_state(ref, mesh, ("u0", "b1f0", "b2f0", "b3f0"))
    mesh.prime(0.0)
    mesh.cycles(cycles)
    expect = mesh.history()
    dev = DeviceArrays(mesh.get("u0"), mesh.get("b1f0"), mesh.get("b2f0"), mesh.get("b3f0"))
    lib = load_library()
    cfg = mesh.cfg
    dx = ((cfg.x1max - cfg.x1min) / cfg.nx1, (cfg.x2max - cfg.x2min) / cfg.nx2, (cfg.x3max - cfg.x3min) / cfg.nx3)
    try:
        for call in range(2):
            out = np.full(10, np.nan)
            rc = lib.chq_history_noalloc(mesh.nx1, mesh.nx2, mesh.nx3, mesh.ng, dx[0], dx[1], dx[2], *dev.ptrs,
                                         out.ctypes.data_as(C.POINTER(C.c_double)), None)
            assert rc == 0, lib.chq_last_error()
            np.testing.assert_allclose(out[:8], expect[:8], rtol=1e-12, atol=1e-14, err_msg=f"call {call}")
            assert abs(out[8] - expect[8]) <= 1e-15, (call, out[8], expect[8])
            np.testing.assert_allclose(out[9], expect[9], rtol=1e-10, atol=1e-16, err_msg=f"call {call}")
    finally:
        dev.free()


def test_noalloc_rejects_meshes_beyond_its_scratch():
    from chasqui_b200 import load_library
    lib = load_library()
    out = np.zeros(10)
    one = C.c_void_p(1)
    # nx3 * ceil(nx2 / 128) = 4097 * 2 > 8192
    rc = lib.chq_history_noalloc(8, 256, 4097, 3, 1.0, 1.0, 1.0, one, one, one, one,
                                 out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == -1
    assert b"too large" in lib.chq_last_error()
