"""Whole-cycle parity on ragged mesh shapes: odd and prime extents that fill no warp, tile or
march evenly, very thin and elongated meshes, and ghost layers deeper than the scheme needs
(mesh.nghost, src/main.cpp:166-168). The device path pads rows to its pitch and cuts its
launch grids to these extents; the result must still match the reference's own loop.

Tolerance as for the other cycle tests (FP64 form): relative L1 <= 1e-12 per field after ten
cycles, the same clock, FOFC count and dt reduction."""
import pytest

from tests import cases
from tests.parity import copy_state, l1_rel, make_pair

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")

SHAPES = {
    "blast3d_17x13x11": (cases.blast(16), ["mesh.nx1=17", "mesh.nx2=13", "mesh.nx3=11"]),
    "blast3d_strong_31x9x7_fofc": (cases.blast(16), ["mesh.nx1=31", "mesh.nx2=9", "mesh.nx3=7",
                                                     "problem.pres_in=1e4", "problem.pres_out=1e-3",
                                                     "time.cfl=0.5"]),
    "ot2d_33x47": (cases.ot(32), ["mesh.nx1=33", "mesh.nx2=47"]),
    "ot2d_97x5": (cases.ot(32), ["mesh.nx1=97", "mesh.nx2=5"]),
    "cpaw2d_wenoz_ng5": (cases.cpaw2d(24), ["mesh.nghost=5"]),
    "shock1d_127_ng4": (cases.shock_tube(128), ["mesh.nx1=127", "mesh.nghost=4"]),
    "loop3d_40x6x4_plm": (cases.field_loop(16, 8), ["mesh.nx1=40", "mesh.nx2=6", "mesh.nx3=4",
                                                    "mhd.reconstruct=plm"]),
    "blast3d_5x67x3_dc_hlle": (cases.blast(16), ["mesh.nx1=5", "mesh.nx2=67", "mesh.nx3=3",
                                                 "mhd.reconstruct=dc", "mhd.rsolver=hlle"]),
}


def _ten_cycles(ref, step):
    for _ in range(10):
        ref.cycles(1)
        step()


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SHAPES))
def test_ragged_shapes_match_reference(name):
    text, ov = SHAPES[name]
    ref, mesh = make_pair(text, ov)
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    assert mesh.clock()["min_dt"] == pytest.approx(ref.min_dt, rel=1e-15)
    _ten_cycles(ref, lambda: mesh.cycles(1))
    ck = mesh.clock()
    assert ck["cycle"] == ref.cycle and ck["t"] == pytest.approx(ref.time, rel=1e-14, abs=0)
    errs = {f: l1_rel(mesh.get(f), ref.get(f)) for f in FIELDS}
    assert max(errs.values()) <= 1e-12, errs
    assert mesh.counters()[0] == ref.fofc_count
    mesh.close()
    ref.close()


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_ragged_shapes_port_matches_reference_bitwise(name):
    """CPU: the oracle's C restatement follows the reference on the same shapes, bit for bit."""
    import numpy as np

    from chasqui_b200.params import Params, config_from_params
    from oracle import portsim, refsim
    if not (portsim.available() and refsim.available()):
        pytest.skip("oracle not built")
    text, ov = SHAPES[name]
    ref = refsim.RefSim(text, ov)
    pin = Params().read_text(text)
    for o in ov:
        pin.override(o)
    port = portsim.PortSim(portsim.cfg_from_chq(config_from_params(pin)))
    for f in FIELDS:
        port.set(f, ref.get(f))
    port.prime(0.0)
    _ten_cycles(ref, lambda: port.cycles(1))
    for f in FIELDS:
        assert np.array_equal(port.get(f), ref.get(f).ravel()), f
    ck = port.clock()
    assert ck["t"] == ref.time and ck["fofc"] == ref.fofc_count
    assert np.all(np.isfinite(ref.get("u0")))
    port.close()
    ref.close()
