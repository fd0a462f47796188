"""Pins the oracle's C restatement (oracle/port) against the reference's own kernels
(oracle/_ref): whole cycles on the same initial states must agree bit for bit (both are
compiled without multiply-add contraction and call the same libm). The cases cover the ideal
path, explicit diffusion inside the stage (src/diffusion.hpp), RKL2 super-time-stepping
(src/sts.hpp), gravity and cooling (src/srcterms.hpp), each alone and combined. CPU only."""
import numpy as np
import pytest

from chasqui_b200.params import Params, config_from_params
from tests import cases
from tests.conftest import ROOT  # noqa: F401

STRONG = ["problem.pres_in=1e4", "problem.pres_out=1e-3", "time.cfl=0.5"]
GRAV_U = ["gravity.uniform=true", "gravity.g1=0.5", "gravity.g2=-0.25", "gravity.g3=1.0"]
GRAV_P = ["gravity.point_mass=true", "gravity.gm=0.05", "gravity.x0=0.05", "gravity.y0=-0.1", "gravity.z0=0.02",
          "gravity.rsoft=0.05"]

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
    # explicit diffusion inside the stage, one coefficient per axis and all three together
    "eta_z": (cases.diffusion("b", 3), ["diffusion.eta=0.02"]),
    "nu_y": (cases.diffusion("v", 2), ["diffusion.nu=0.02"]),
    "kappa_x": (cases.diffusion("temp", 1), ["diffusion.kappa=0.003"]),
    "blast3d_all_diffusion_fofc": (cases.blast(12), STRONG + ["diffusion.nu=1e-3", "diffusion.kappa=1e-3",
                                                             "diffusion.eta=1e-3"]),
    # RKL2 after the hyperbolic step
    "eta_y_sts": (cases.diffusion("b", 2), ["diffusion.eta=0.1", "diffusion.sts=true"]),
    "ot2d_all_sts": (cases.ot(24), ["diffusion.nu=0.05", "diffusion.kappa=0.05", "diffusion.eta=0.05",
                                    "diffusion.sts=true"]),
    "blast3d_sts_fofc": (cases.blast(12), STRONG + ["diffusion.nu=5e-3", "diffusion.eta=5e-3", "diffusion.sts=true"]),
    # gravity (uniform and point mass) and cooling (alpha = 1, alpha != 1 with the floor)
    "point_mass_blast_fofc": (cases.blast(12), GRAV_P + STRONG),
    "ot2d_uniform_gravity": (cases.ot(24), GRAV_U),
    "ot2d_cooling_alpha_one": (cases.ot(24), ["cooling.enabled=true", "cooling.lambda0=0.5"]),
    "blast3d_cooling_floor": (cases.blast(12), ["cooling.enabled=true", "cooling.lambda0=5.0", "cooling.alpha=2.0",
                                                "cooling.tfloor=0.05"]),
    "ot2d_cooling_gravity_diffusion": (cases.ot(24), GRAV_U + ["cooling.enabled=true", "cooling.lambda0=0.2",
                                                               "diffusion.nu=2e-3", "diffusion.kappa=2e-3"]),
    "ot2d_cooling_sts": (cases.ot(24), ["cooling.enabled=true", "cooling.lambda0=0.2", "diffusion.eta=0.02",
                                        "diffusion.sts=true"]),
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
    assert ck["min_dt"] == ref.min_dt and port.sts_stages() == ref.sts_stages
    np.testing.assert_allclose(port.history(), ref.history(), rtol=1e-12, atol=1e-15)
