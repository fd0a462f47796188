"""Explicit diffusion and RKL2 super-time-stepping against the reference's own loop.

Covers viscosity, thermal conduction and Ohmic resistivity added inside each RK stage
(src/main.cpp:53-70, src/diffusion.hpp), the parabolic limit joining the time step
(src/main.cpp:239, 280), the diffusive fluxes re-added by the FOFC repair (src/fofc.hpp:89-93)
and the operator-split RKL2 advance (src/sts.hpp:109-158, src/main.cpp:282-290).

Tolerance (FP64 form): relative L1 <= 1e-12 per field after 10 cycles, as for the ideal
cycles (only pow(rho, gamma) in the entropy slot rounds differently on the device); the
cycle count, clock, FOFC count and RKL2 stage count must match exactly.
"""
import numpy as np
import pytest

from tests import cases
from tests.parity import copy_state, l1_rel, make_pair

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")

ALL3 = ["diffusion.nu=2e-3", "diffusion.kappa=2e-3", "diffusion.eta=2e-3"]
STRONG_BLAST = ["problem.pres_in=1e4", "problem.pres_out=1e-3", "time.cfl=0.5"]

CASES = {
    # the reference's decay tests (tests/physics.sh), one per coefficient and axis
    "eta_x": (cases.diffusion("b", 1), ["diffusion.eta=0.02"]),
    "eta_y": (cases.diffusion("b", 2), ["diffusion.eta=0.02"]),
    "eta_z": (cases.diffusion("b", 3), ["diffusion.eta=0.02"]),
    "nu_y": (cases.diffusion("v", 2), ["diffusion.nu=0.02"]),
    "nu_z": (cases.diffusion("v", 3), ["diffusion.nu=0.02"]),
    "kappa_x": (cases.diffusion("temp", 1), ["diffusion.kappa=0.003"]),
    # all three terms on a nonlinear flow, with FOFC, the limiter and other integrators
    "ot2d_all": (cases.ot(32), ALL3),
    "ot2d_all_rk2_limiter": (cases.ot(32), ALL3 + ["time.integrator=rk2", "mhd.flux_limiter=true"]),
    "blast3d_all_fofc": (cases.blast(16), STRONG_BLAST + ["diffusion.nu=1e-3", "diffusion.kappa=1e-3",
                                                         "diffusion.eta=1e-3"]),
    # RKL2 super-time-stepping
    "eta_y_sts": (cases.diffusion("b", 2), ["diffusion.eta=0.1", "diffusion.sts=true"]),
    "kappa_x_sts": (cases.diffusion("temp", 1), ["diffusion.kappa=0.02", "diffusion.sts=true"]),
    "ot2d_all_sts": (cases.ot(32), ["diffusion.nu=0.05", "diffusion.kappa=0.05", "diffusion.eta=0.05",
                                    "diffusion.sts=true"]),
    "blast3d_sts_fofc": (cases.blast(16), STRONG_BLAST + ["diffusion.nu=5e-3", "diffusion.eta=5e-3",
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
        assert ck["t"] == pytest.approx(ref.time, rel=1e-14, abs=0)
    errs = {f: l1_rel(mesh.get(f), ref.get(f)) for f in FIELDS}
    assert max(errs.values()) <= 1e-12, errs
    assert mesh.counters()[0] == ref.fofc_count
    assert mesh.sts_stages() == ref.sts_stages


def test_cases_exercise_what_they_name():
    """The STS cases take more than the minimum two RKL2 stages and the diffusive blast
    triggers first-order corrections, so both the recursion and the repair path run."""
    text, ov = CASES["ot2d_all_sts"]
    ref, _ = make_pair(text, ov)
    ref.cycles(3)
    assert ref.sts_stages > 2 * 3
    text, ov = CASES["blast3d_all_fofc"]
    ref, _ = make_pair(text, ov)
    ref.cycles(10)
    assert ref.fofc_count > 0


def test_mixed_form_tracks_reference():
    """Mixed form (FP32 primitives, fluxes and EMFs; FP64 state): smooth diffusive flow stays
    within 1e-4 relative L1 of the FP64 reference after 10 cycles."""
    text, ov = CASES["ot2d_all"]
    ref, mesh = make_pair(text, ov, precision="mixed")
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    ref.cycles(10)
    mesh.cycles(10)
    u_ref, u_dev = ref.get("u0"), mesh.get("u0")
    for n in range(5):
        assert l1_rel(u_dev[n], u_ref[n]) <= 1e-4, n


def test_decay_rate_matches_exact_solution():
    """Resistive decay of a sinusoid: B(t) = B(0) exp(-eta k^2 t) (tests/physics.sh)."""
    text, ov = CASES["eta_x"]
    ref, mesh = make_pair(text, ov)
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    ng = mesh.ng
    act = (1, 0, 0, slice(ng, ng + mesh.nx1))   # cell-centred B_y over the active cells
    b0 = mesh.get("bcc")[act].copy()
    while mesh.clock()["t"] < 0.5:
        mesh.cycles(16)
    t = mesh.clock()["t"]
    b1 = mesh.get("bcc")[act]
    k = 2 * np.pi
    ratio = np.max(np.abs(b1)) / np.max(np.abs(b0))
    assert ratio == pytest.approx(np.exp(-0.02 * k * k * t), rel=2e-3)


def test_batch_groups_diffusion_by_switch():
    """Explicit diffusion and RKL2 meshes batch (tests/test_batch.py checks the results), each
    only with meshes that have the same switches."""
    from chasqui_b200 import Batch, ChqError
    text, ov = CASES["ot2d_all"]
    _, mesh = make_pair(text, ov)
    Batch([mesh]).close()
    _, plain = make_pair(text, [])
    with pytest.raises(ChqError):
        Batch([mesh, plain])
    _, sts = make_pair(text, list(ov) + ["diffusion.sts=true"])
    Batch([sts]).close()
    with pytest.raises(ChqError):
        Batch([mesh, sts])
