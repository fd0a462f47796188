"""Non-stalling output snapshots (chq_snapshot): the copy taken behind the queued work equals
a synchronous download of the same cycle's state, in both precision forms, while cycles
queued after it run on; a second snapshot waits for the first."""
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
