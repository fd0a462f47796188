"""Non-stalling output snapshots (chq_snapshot): the copy taken behind the queued work equals
a synchronous download of the same cycle's state, in both precision forms, while cycles
queued after it run on; a second snapshot waits for the first. The "vtk" field is the cell
data of the reference's VTK dump (src/output.hpp:71-84) built on the device."""
import numpy as np
import pytest

from tests import cases
from tests.parity import copy_state, make_pair

pytestmark = pytest.mark.gpu

NAMES = ["u0", "b1f0", "b2f0", "b3f0", "w", "bcc"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_snapshot_equals_download_of_that_cycle(precision):
    ref, a = make_pair(cases.blast(20), [], precision=precision)
    _, b = make_pair(cases.blast(20), [], precision=precision)
    for m in (a, b):
        copy_state(ref, m, ("u0", "b1f0", "b2f0", "b3f0"))
        m.prime(0.0)
        m.cycles(3)
    a.snapshot(NAMES)
    a.cycles(4)              # queued after the snapshot: must not leak into it
    snap = a.snapshot_wait()
    want = {n: b.get(n) for n in NAMES}
    for n in NAMES:
        assert np.array_equal(snap[n], want[n]), n
    b.cycles(4)
    for n in ("u0", "b2f0"):
        assert np.array_equal(a.get(n), b.get(n)), n
    # back-to-back snapshots: the second waits for the first
    a.snapshot(["u0"])
    a.snapshot(["b1f0"])
    assert np.array_equal(a.snapshot_wait()["b1f0"], a.get("b1f0"))


VTK_CASES = {"blast3d_20": (cases.blast(20), []), "ot2d_33x47": (cases.ot(32), ["mesh.nx1=33", "mesh.nx2=47"]),
             "shock1d_64": (cases.shock_tube(64), [])}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", sorted(VTK_CASES))
def test_vtk_cells_are_the_reference_dump_payload(precision, case):
    """rho, prs, vx1..3, Bx1..3 over the active cells, i fastest, rounded to float and stored
    big-endian: bit for bit what the reference's writer makes of the same w and bcc."""
    text, ov = VTK_CASES[case]
    ref, m = make_pair(text, ov, precision=precision)
    copy_state(ref, m, ("u0", "b1f0", "b2f0", "b3f0"))
    m.prime(0.0)
    m.cycles(2)
    m.snapshot(["vtk"])
    cells = m.snapshot_wait()["vtk"]
    w, bcc = m.get("w"), m.get("bcc")
    ks = m.ng if m.nx3 > 1 else 0
    js = m.ng if m.nx2 > 1 else 0
    act = (slice(ks, ks + m.nx3), slice(js, js + m.nx2), slice(m.ng, m.ng + m.nx1))
    planes = [w[0], w[4], w[1], w[2], w[3], bcc[0], bcc[1], bcc[2]]
    want = b"".join(np.ascontiguousarray(p[act]).astype(">f4").tobytes() for p in planes)
    got = cells.tobytes()
    assert len(got) == len(want) == 32 * m.nx1 * m.nx2 * m.nx3
    assert got == want
    m.close()
    ref.close()
