"""Pins the oracle's C restatement (oracle/port) against the reference's own kernels
(oracle/_ref): whole cycles on the same initial states must agree bit for bit (both are
compiled without multiply-add contraction and call the same libm). CPU only."""
import numpy as np
import pytest

from chasqui_b200.params import Params, config_from_params
from tests import cases
from tests.conftest import ROOT  # noqa: F401

CASES = {
    "ot2d_ppm_hlld": (cases.ot(32), []),
    "blast3d_ppm_hlld": (cases.blast(12), []),
    "cpaw2d_wenoz": (cases.cpaw2d(24), []),
    "shock1d_plm_hlle": (cases.shock_tube(64), ["mhd.reconstruct=plm", "mhd.rsolver=hlle"]),
    "loop3d_ppmx_lhlld_char": (cases.field_loop(12, 6), ["mhd.rsolver=lhlld", "mhd.characteristic=true"]),
    "ot2d_dc_rk4_lowmach_dual": (cases.ot(24), ["mhd.reconstruct=dc", "time.integrator=rk4", "mhd.low_mach=true",
                                                "mhd.dual_energy=true"]),
    "ot2d_rk2_limiter": (cases.ot(24), ["time.integrator=rk2", "mhd.flux_limiter=true"]),
    "blast3d_strong_fofc_reflect": (cases.blast(12), ["problem.pres_in=1e4", "problem.pres_out=1e-3", "time.cfl=0.5",
                                                      "mesh.bc_x1=reflect", "mesh.bc_x3=outflow"]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_port_matches_reference_bitwise(name):
    from oracle import portsim, refsim
    if not (portsim.available() and refsim.available()):
        pytest.skip("oracle not built")
    text, ov = CASES[name]
    ref = refsim.RefSim(text, ov)
    pin = Params().read_text(text)
    for o in ov:
        pin.override(o)
    port = portsim.PortSim(portsim.cfg_from_chq(config_from_params(pin)))
    for f in ("u0", "b1f0", "b2f0", "b3f0"):
        port.set(f, ref.get(f))
    port.prime(0.0)
    assert port.clock()["min_dt"] == ref.min_dt
    for _ in range(6):
        ref.cycles(1)
        port.cycles(1)
    for f in ("u0", "u1", "b1f0", "b2f0", "b3f0", "w", "bcc", "ecc", "f1", "f2", "f3", "e1", "e2", "e3"):
        a, b = port.get(f), ref.get(f).ravel()
        assert np.array_equal(a, b), (f, float(np.max(np.abs(a - b))))
    ck = port.clock()
    assert ck["t"] == ref.time and ck["cycle"] == ref.cycle and ck["fofc"] == ref.fofc_count
    np.testing.assert_allclose(port.history(), ref.history(), rtol=1e-12, atol=1e-15)
