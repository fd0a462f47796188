"""Golden fixtures written by the reference itself (tests/golden/make_golden.py runs the
reference's own kernels, compiled in place, on each case's input file): the initial state,
the state after N cycles, the clock, the FOFC count and the history sums.

CPU: the fixtures agree with the reference when it is built here (re-run, bit for bit), and
the project's C restatement of the path (oracle/port) reproduces every fixture bit for bit,
including those with diffusion, RKL2 and source terms. GPU: the device path reproduces every fixture (relative L1 <= 1e-12 per field, the
same clock and FOFC count) with no reference present at run time."""
import glob
import os

import numpy as np
import pytest

from chasqui_b200.params import Params, config_from_params
from tests.conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
NAMES = [os.path.basename(f)[:-4] for f in FILES]
FIELDS = ("u0", "b1f0", "b2f0", "b3f0")


def _load(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    ov = [o for o in d["overrides"].tolist() if o]
    return d, str(d["text"]), ov


def _pin(text, ov):
    pin = Params().read_text(text)
    for o in ov:
        pin.override(o)
    return pin


def test_fixtures_present():
    assert len(NAMES) >= 7
    for name in NAMES:
        d, _, _ = _load(name)
        assert int(d["cycle"]) == int(d["cycles"]) > 0
        for f in FIELDS:
            assert d["in_" + f].shape == d["out_" + f].shape and np.isfinite(d["out_" + f]).all()
        assert not np.array_equal(d["in_u0"], d["out_u0"])


@pytest.mark.parametrize("name", NAMES)
def test_fixture_is_the_reference_output(name):
    from oracle.refsim import RefSim, available
    if not available():
        pytest.skip("the reference build (oracle/_ref) is not here")
    d, text, ov = _load(name)
    ref = RefSim(text, ov)
    for f in FIELDS:
        assert np.array_equal(ref.get(f), d["in_" + f]), f
    ref.cycles(int(d["cycles"]))
    for f in FIELDS:
        assert np.array_equal(ref.get(f), d["out_" + f]), f
    assert ref.time == float(d["time"]) and ref.fofc_count == int(d["fofc"])
    ref.close()


@pytest.mark.parametrize("name", NAMES)
def test_port_reproduces_fixture_bitwise(name):
    from oracle import portsim
    if not portsim.available():
        pytest.skip("oracle/_port not built")
    d, text, ov = _load(name)
    port = portsim.PortSim(portsim.cfg_from_chq(config_from_params(_pin(text, ov))))
    for f in FIELDS:
        port.set(f, d["in_" + f])
    port.prime(0.0)
    port.cycles(int(d["cycles"]))
    for f in FIELDS:
        assert np.array_equal(port.get(f), d["out_" + f].ravel()), f
    ck = port.clock()
    assert ck["t"] == float(d["time"]) and ck["cycle"] == int(d["cycle"]) and ck["fofc"] == int(d["fofc"])
    port.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_device_reproduces_fixture(name):
    from chasqui_b200 import Mesh, make_config
    d, text, ov = _load(name)
    mesh = Mesh(make_config(**config_from_params(_pin(text, ov))))
    for f in FIELDS:
        mesh.set(f, d["in_" + f])
    mesh.prime(0.0)
    mesh.cycles(int(d["cycles"]))
    ck = mesh.clock()
    assert ck["cycle"] == int(d["cycle"])
    assert ck["t"] == pytest.approx(float(d["time"]), rel=1e-14, abs=0)
    for f in FIELDS:
        a, b = mesh.get(f), d["out_" + f]
        err = float(np.sum(np.abs(a - b))) / max(float(np.sum(np.abs(b))), 1e-300)
        assert err <= 1e-12, (f, err)
    assert mesh.counters()[0] == int(d["fofc"])
    np.testing.assert_allclose(mesh.history(), d["history"], rtol=1e-12, atol=1e-14)
    mesh.close()
