"""Gravity and cooling source terms against the reference's own loop.

Gravity (src/srcterms.hpp:10-41) is applied after every Update and after the FOFC re-run
(src/main.cpp:76, 89), here as the epilogue of the update kernel; cooling (src/srcterms.hpp:
43-71) is operator split after the step with its own con2prim and boundary fill
(src/main.cpp:282-290). FP64 tolerance: relative L1 <= 1e-12 per field after 10 cycles
(cooling uses exp / pow, which round differently on the device by at most an ulp or two);
the reference's exact-solution checks of tests/physics.sh are repeated on the device."""
import math

import numpy as np
import pytest

from tests import cases
from tests.parity import copy_state, l1_rel, make_pair

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")

UNIFORM = """
[mesh]
nx1 = 16
nx2 = 16
nx3 = 16
[time]
tlim = 1.0
[mhd]
reconstruct = plm
[problem]
name = uniform
dens = 2.0
pres = 1.0
"""

GRAV_U = ["gravity.uniform=true", "gravity.g1=0.5", "gravity.g2=-0.25", "gravity.g3=1.0"]
GRAV_P = ["gravity.point_mass=true", "gravity.gm=0.05", "gravity.x0=0.05", "gravity.y0=-0.1", "gravity.z0=0.02",
          "gravity.rsoft=0.05"]

CASES = {
    "uniform_gravity": (UNIFORM, GRAV_U),
    "point_mass_blast_fofc": (cases.blast(16), GRAV_P + ["problem.pres_in=1e4", "problem.pres_out=1e-3",
                                                        "time.cfl=0.5"]),
    "point_mass_ot2d_uniform_too": (cases.ot(32), GRAV_P + GRAV_U),
    "cooling_alpha_half": (UNIFORM, ["cooling.enabled=true", "cooling.lambda0=0.1", "cooling.alpha=0.5"]),
    "cooling_alpha_one_ot2d": (cases.ot(32), ["cooling.enabled=true", "cooling.lambda0=0.5"]),
    "cooling_floor_blast": (cases.blast(16), ["cooling.enabled=true", "cooling.lambda0=5.0", "cooling.alpha=2.0",
                                             "cooling.tfloor=0.05"]),
    "cooling_gravity_diffusion": (cases.ot(32), GRAV_U + ["cooling.enabled=true", "cooling.lambda0=0.2",
                                                         "diffusion.nu=2e-3", "diffusion.kappa=2e-3"]),
    "cooling_with_sts": (cases.ot(32), ["cooling.enabled=true", "cooling.lambda0=0.2", "diffusion.eta=0.02",
                                        "diffusion.sts=true"]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_ten_cycles_match_reference(name):
    text, ov = CASES[name]
    ref, mesh = make_pair(text, ov)
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    assert mesh.clock()["min_dt"] == pytest.approx(ref.min_dt, rel=1e-15)
    for c in range(10):
        ref.cycles(1)
        mesh.cycles(1)
        ck = mesh.clock()
        assert ck["cycle"] == ref.cycle
        assert ck["t"] == pytest.approx(ref.time, rel=1e-13, abs=0)
    errs = {f: l1_rel(mesh.get(f), ref.get(f)) for f in FIELDS}
    assert max(errs.values()) <= 1e-12, errs
    assert mesh.counters()[0] == ref.fofc_count


def _run_to(mesh, t_end):
    while mesh.clock()["t"] < t_end - 1e-12:
        mesh.cycles(32)


def test_uniform_gravity_momentum_is_exact():
    """momentum = rho g t V (tests/physics.sh): uniform state, uniform field, t = 1."""
    ref, mesh = make_pair(UNIFORM, GRAV_U)
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    _run_to(mesh, 1.0)
    h = mesh.history()
    assert h[1] == pytest.approx(1.0, rel=1e-9)     # 2.0 * 0.5 * 1.0 * V
    assert h[3] == pytest.approx(2.0, rel=1e-9)


def test_cooling_temperature_is_exact():
    """T(t) = (T0^(1-a) - (a-1) c t)^(1/(1-a)) for a = 1/2 (tests/physics.sh)."""
    ref, mesh = make_pair(UNIFORM, ["cooling.enabled=true", "cooling.lambda0=0.1", "cooling.alpha=0.5"])
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    _run_to(mesh, 1.0)
    w = mesh.get("w")
    ng = mesh.ng
    act = (slice(ng, -ng),) * 3
    T = float(np.mean(w[4][act] / w[0][act]))
    c = (5.0 / 3.0 - 1.0) * 2.0 * 0.1
    assert T == pytest.approx((math.sqrt(0.5) - 0.5 * c) ** 2, rel=1e-6)


def test_batch_groups_source_terms_by_switch():
    """A batch takes meshes with gravity (or cooling) only together with meshes that have it
    too; their coefficients may differ (tests/test_batch.py checks the results)."""
    from chasqui_b200 import Batch, ChqError
    _, grav = make_pair(UNIFORM, GRAV_U)
    _, plain = make_pair(UNIFORM, [])
    _, cool = make_pair(UNIFORM, ["cooling.enabled=true", "cooling.lambda0=0.1"])
    Batch([grav]).close()
    for pair in ([grav, plain], [grav, cool], [cool, plain]):
        with pytest.raises(ChqError):
            Batch(pair)
