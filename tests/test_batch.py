"""Batched stepping (chq_batch): many meshes of one class advanced with one launch per kernel
kind per stage. Every member must end bit for bit where it ends when stepped alone, with or
without CUDA-graph replay, including members that reach their end time at different cycles."""
import numpy as np
import pytest

from chasqui_b200 import Batch, ChqError, Mesh, Params, config_from_params, make_config
from tests import cases

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")


def _mesh(text, ov=(), precision="fp64"):
    from oracle.refsim import RefSim
    ref = RefSim(text, list(ov))
    pin = Params().read_text(text)
    for o in ov:
        pin.override(o)
    pin.override(f"mhd.precision={precision}")
    m = Mesh(make_config(**config_from_params(pin)))
    for f in FIELDS:
        m.set(f, ref.get(f))
    m.prime(0.0)
    ref.close()
    return m


SETS = {
    "mixed_dims_fp64": [(cases.ot(32), ()), (cases.blast(16), ()), (cases.ot(48), ("problem.name=orszag_tang",)),
                        (cases.cpaw3d_extruded(16, 8), ("mhd.reconstruct=ppm",))],
    "wenoz_mixed_precision": [(cases.cpaw2d(32), ()), (cases.cpaw3d_extruded(16, 8), ()),
                              (cases.blast(12), ("mhd.reconstruct=wenoz",))],
}


@pytest.mark.parametrize("graph", [False, True], ids=["launches", "graph"])
@pytest.mark.parametrize("name", sorted(SETS))
def test_batched_members_equal_solo(name, graph):
    prec = "mixed" if "mixed_precision" in name else "fp64"
    specs = SETS[name]
    solo = [_mesh(t, ov, prec) for t, ov in specs]
    for m in solo:
        m.cycles(7)
    expect = [{f: m.get(f) for f in FIELDS} for m in solo]
    clocks = [m.clock() for m in solo]
    members = [_mesh(t, ov, prec) for t, ov in specs]
    b = Batch(members, graph=graph)
    b.cycles(3)
    b.cycles(4)
    st = b.status()
    for j, m in enumerate(members):
        assert st[j]["cycle"] == 7 and st[j]["t"] == clocks[j]["t"], (j, st[j], clocks[j])
        for f in FIELDS:
            assert np.array_equal(m.get(f), expect[j][f]), (name, j, f)
    assert b.kernel_launches() > 0
    b.close()


def test_members_stop_at_their_own_tlim():
    specs = [(cases.ot(32), ("time.tlim=0.004",)), (cases.ot(40), ("time.tlim=0.5",))]
    solo = [_mesh(t, ov) for t, ov in specs]
    for m in solo:
        m.cycles(12)
    members = [_mesh(t, ov) for t, ov in specs]
    b = Batch(members, graph=True)
    b.cycles(12)
    st = b.status()
    assert st[0]["done"] or st[0]["t"] == pytest.approx(0.004, abs=0)
    assert st[0]["cycle"] < 12 and st[1]["cycle"] == 12
    for j in range(2):
        assert st[j]["cycle"] == solo[j].clock()["cycle"]
        assert np.array_equal(members[j].get("u0"), solo[j].get("u0"))


def test_batch_rejects_mixed_classes():
    a = _mesh(cases.ot(16))
    c = _mesh(cases.ot(16), ("mhd.reconstruct=wenoz",))
    with pytest.raises(ChqError):
        Batch([a, c])
    with pytest.raises(ChqError):
        Batch([a, a])
