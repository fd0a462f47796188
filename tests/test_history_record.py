"""Device-recorded .hst rows (chq_history_record / chq_history_drain).

The reference writes a history row after every cycle whose new time reaches the next output
time (t >= next_hst - eps after t += dt, then next_hst += dt_hst; src/main.cpp:212-223,
output::History src/output.hpp:91-119). Here the test runs on the device, the sums ride on
the con2prim of the cycle's final state, and the rows collect in a ring. Checked against a
twin mesh stepped one cycle at a time with that host-side test and chq_history(): the same
rows at the same cycles (t, dt and divB_max bit for bit, the sums to their reduction-order
rounding), on the graph-replayed ideal path, the mixed form, FOFC, cooling and RKL2."""
import numpy as np
import pytest

from chasqui_b200 import ChqError
from tests import cases
from tests.parity import copy_state, make_pair

STRONG = ["problem.pres_in=1e4", "problem.pres_out=1e-3", "time.cfl=0.5"]

CASES = {
    "ot2d_fp64": (cases.ot(32), [], "fp64"),
    "ot2d_mixed": (cases.ot(32), [], "mixed"),
    "blast3d_fofc_fp64": (cases.blast(16), STRONG, "fp64"),
    "ot2d_cooling_fp64": (cases.ot(24), ["cooling.enabled=true", "cooling.lambda0=0.2"], "fp64"),
    "eta_y_sts_fp64": (cases.diffusion("b", 2), ["diffusion.eta=0.1", "diffusion.sts=true"], "fp64"),
}


def _twins(text, ov, prec):
    ref, a = make_pair(text, ov, precision=prec)
    _, b = make_pair(text, ov, precision=prec)
    copy_state(ref, a)
    copy_state(ref, b)
    ref.close()
    a.prime(0.0)
    b.prime(0.0)
    return a, b


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_recorded_rows_match_host_output_test(name):
    text, ov, prec = CASES[name]
    a, b = _twins(text, ov, prec)
    cfl = 0.5 if "time.cfl=0.5" in ov else 0.4
    dt_hst = 1.7 * cfl * a.clock()["min_dt"]   # an output about every other cycle
    eps = 1e-10
    ncyc = 16
    a.record_history(dt_hst, dt_hst, eps, capacity=64)
    a.cycles(ncyc)
    rows, lost, nxt = a.drain_history(64)

    expect, nxt_b = [], dt_hst
    for _ in range(ncyc):
        b.cycles(1)
        ck = b.clock()
        if ck["t"] >= nxt_b - eps:
            expect.append([ck["t"], ck["dt"]] + list(b.history()))
            nxt_b += dt_hst
    E = np.array(expect)
    assert lost == 0 and len(rows) == len(E) >= 3, (len(rows), len(E))
    assert np.array_equal(rows[:, :2], E[:, :2])
    assert np.array_equal(rows[:, 10], E[:, 10])   # divB_max: a max, order independent
    scale = np.maximum(1.0, np.abs(E).max(axis=0))
    err = np.abs(rows - E) / scale
    assert float(err.max()) <= 1e-12, err.max(axis=0)
    assert nxt == nxt_b
    # the recorded state is the stepped state: both meshes end bit for bit equal
    for f in ("u0", "b1f0", "b2f0", "b3f0"):
        assert np.array_equal(a.get(f), b.get(f)), f
    a.close()
    b.close()


@pytest.mark.gpu
def test_ring_counts_lost_rows_and_turns_off():
    a, b = _twins(cases.ot(16), [], "fp64")
    b.close()
    a.record_history(1e-12, 0.0, 0.0, capacity=3)   # every cycle is an output
    a.cycles(5)
    rows, lost, _ = a.drain_history(8)
    assert len(rows) == 3 and lost == 2
    a.cycles(2)
    first, lost, _ = a.drain_history(1)   # the second row stays in the ring
    assert len(first) == 1 and lost == 0
    second, lost, _ = a.drain_history(8)
    assert len(second) == 1 and lost == 0 and second[0, 0] > first[0, 0]
    a.record_history(0.0, 0.0, 0.0, capacity=0)
    with pytest.raises(ChqError):
        a.drain_history()
    with pytest.raises(ChqError):
        a.record_history(0.0, 0.0, 0.0, capacity=4)   # an interval is required
    a.close()
