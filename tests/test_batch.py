"""Batched stepping (chq_batch): many meshes of one class advanced with one launch per kernel
kind per stage. In the FP64 form every member must end bit for bit where it ends when stepped
alone, with or without CUDA-graph replay, including members that reach their end time at
different cycles. In the mixed form the batched and the single-mesh flux kernels are two
FP32 instantiations whose multiply-adds the compiler may fuse differently, so a member must
end bit for bit where it ends in a batch of its own (its result never depends on its
batch-mates) and within the FP32 rounding growth of the single-mesh run (2e-3 relative L1 after
7 cycles, set by a strong blast whose FOFC switches amplify rounding; the same order as the
mixed form's distance from FP64)."""
import numpy as np
import pytest

from chasqui_b200 import Batch, ChqError, Mesh, Params, config_from_params, make_config
from tests import cases
from tests.parity import l1_rel

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
    # odd and prime extents side by side: each member's blocks cut to its own shape
    "ragged_shapes_fp64": [(cases.blast(16), ("mesh.nx1=17", "mesh.nx2=13", "mesh.nx3=11")),
                           (cases.ot(32), ("mesh.nx1=33", "mesh.nx2=47")), (cases.ot(32), ("mesh.nx1=97", "mesh.nx2=5")),
                           (cases.blast(16), ("mesh.nx1=31", "mesh.nx2=9", "mesh.nx3=7", "problem.pres_in=1e4",
                                              "problem.pres_out=1e-3", "time.cfl=0.5"))],
}


GRAV_U = ("gravity.uniform=true", "gravity.g1=0.5", "gravity.g2=-0.25", "gravity.g3=1.0")
GRAV_P = ("gravity.point_mass=true", "gravity.gm=0.05", "gravity.x0=0.05", "gravity.y0=-0.1", "gravity.z0=0.02",
          "gravity.rsoft=0.05")
STRONG = ("problem.pres_in=1e4", "problem.pres_out=1e-3", "time.cfl=0.5")

# explicit diffusion, gravity and cooling: every member has the terms on, with its own
# coefficients; the strong blasts add FOFC re-runs (diffusive fluxes re-added on repaired faces)
SETS.update({
    "diffusion_fp64": [(cases.ot(32), ("diffusion.nu=2e-3", "diffusion.kappa=2e-3", "diffusion.eta=1e-3")),
                       (cases.blast(16), STRONG + ("diffusion.eta=2e-3",)),
                       (cases.diffusion("b", 1, 32, 8), ("diffusion.eta=0.01", "mhd.reconstruct=ppm"))],
    "gravity_fp64": [(cases.blast(16), STRONG + GRAV_P), (cases.ot(32), GRAV_P + GRAV_U),
                     (cases.cpaw3d_extruded(16, 8), ("mhd.reconstruct=ppm",) + GRAV_U)],
    "cooling_fp64": [(cases.ot(32), ("cooling.enabled=true", "cooling.lambda0=0.5")),
                     (cases.blast(16), ("cooling.enabled=true", "cooling.lambda0=5.0", "cooling.alpha=2.0",
                                        "cooling.tfloor=0.05"))],
    # RKL2: the hyperbolic stages, then the super-time-stepping stages batched across members
    # with different stage counts (members past their count skip)
    "rkl2_fp64": [(cases.ot(32), ("diffusion.eta=0.2", "diffusion.sts=true")),
                  (cases.diffusion("temp", 1, 32, 8), ("diffusion.kappa=0.2", "diffusion.sts=true",
                                                      "mhd.reconstruct=ppm")),
                  (cases.blast(16), STRONG + ("diffusion.nu=5e-3", "diffusion.eta=5e-3", "diffusion.sts=true"))],
    "rkl2_cooling_fp64": [(cases.ot(32), ("diffusion.eta=0.02", "diffusion.sts=true", "cooling.enabled=true",
                                          "cooling.lambda0=0.2")),
                          (cases.blast(16), ("diffusion.nu=2e-3", "diffusion.sts=true", "cooling.enabled=true",
                                             "cooling.lambda0=1.0"))],
    "rkl2_mixed_precision": [(cases.ot(32), ("diffusion.eta=0.02", "diffusion.sts=true")),
                             (cases.diffusion("b", 2, 32, 8), ("diffusion.eta=0.1", "diffusion.sts=true",
                                                              "mhd.reconstruct=ppm"))],
    "all_terms_fp64": [(cases.ot(32), GRAV_U + ("cooling.enabled=true", "cooling.lambda0=0.2", "diffusion.nu=2e-3",
                                                "diffusion.kappa=2e-3")),
                       (cases.blast(16), STRONG + GRAV_P + ("cooling.enabled=true", "cooling.lambda0=1.0",
                                                            "diffusion.eta=1e-3"))],
})


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
    if prec == "mixed":
        alone = []
        for t, ov in specs:
            m = _mesh(t, ov, prec)
            b1 = Batch([m], graph=graph)
            b1.cycles(7)
            st1 = b1.status()[0]
            alone.append(({f: m.get(f) for f in FIELDS}, st1))
            b1.close()
        for j, m in enumerate(members):
            assert st[j]["cycle"] == 7 and st[j]["t"] == alone[j][1]["t"], (j, st[j], alone[j][1])
            # against the single-mesh run: FP32 rounding differences, which the set's strong
            # blast amplifies to 1e-4..1e-3 within 7 cycles (FOFC switches), as against FP64
            assert st[j]["t"] == pytest.approx(clocks[j]["t"], rel=1e-3)
            got = {f: m.get(f) for f in FIELDS}
            for f in FIELDS:
                assert np.array_equal(got[f], alone[j][0][f]), (name, j, f)
            assert l1_rel(got["u0"], expect[j]["u0"]) <= 2e-3, (name, j)
            # face fields against the norm of the whole field (a component that is pure
            # round-off, like b3 of a field in the x-y plane, has no relative error of its own)
            bnorm = sum(float(np.sum(np.abs(expect[j][f]))) for f in FIELDS[1:])
            for f in FIELDS[1:]:
                assert float(np.sum(np.abs(got[f] - expect[j][f]))) <= 2e-3 * bnorm, (name, j, f)
    else:
        for j, m in enumerate(members):
            assert st[j]["cycle"] == 7 and st[j]["t"] == clocks[j]["t"], (j, st[j], clocks[j])
            for f in FIELDS:
                assert np.array_equal(m.get(f), expect[j][f]), (name, j, f)
            assert m.sts_stages() == solo[j].sts_stages(), (name, j)
        if name == "rkl2_fp64":
            counts = [m.sts_stages() for m in solo]
            assert min(counts) > 0 and len(set(counts)) > 1, counts   # members of unequal stage counts
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
    # source terms, diffusion and RKL2 on in every member or in none
    sts = ("diffusion.eta=1e-3", "diffusion.sts=true")
    for ov in (GRAV_U, ("cooling.enabled=true", "cooling.lambda0=0.5"), ("diffusion.nu=1e-3",), sts):
        with pytest.raises(ChqError):
            Batch([a, _mesh(cases.ot(16), ov)])
    with pytest.raises(ChqError):
        Batch([_mesh(cases.ot(16), ("diffusion.eta=1e-3",)), _mesh(cases.ot(16), sts)])
    Batch([_mesh(cases.ot(16), sts)]).close()
