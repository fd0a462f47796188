"""Kernel-by-kernel parity of the CUDA path (through the C ABI) with the reference's own
kernels (oracle/_ref), on identical full states. FP64 form.

Expected agreement: bitwise for every kernel whose arithmetic is +, -, *, /, sqrt, min/max
(both sides round these correctly and neither contracts multiply-adds). The one exception
is pow(rho, gamma) in con2prim and in the dual-energy branches, where the device and glibc
may round differently; those slots are checked to 1e-14 relative."""
import numpy as np
import pytest

from tests import cases
from tests.parity import STATE_FIELDS, assert_fields, copy_state, make_pair

pytestmark = pytest.mark.gpu

CASES = {
    "ot2d_ppm_hlld": (cases.ot(32), []),
    "blast3d_ppm_hlld": (cases.blast(16), []),
    "cpaw2d_wenoz_hlld": (cases.cpaw2d(32), []),
    "cpaw3d_ppmx_lhlld": (cases.cpaw3d_extruded(16, 8), ["mhd.reconstruct=ppmx", "mhd.rsolver=lhlld"]),
    "shock1d_plm_hlle": (cases.shock_tube(64), ["mhd.reconstruct=plm", "mhd.rsolver=hlle"]),
    "shock1d_dc_hlld": (cases.shock_tube(48), ["mhd.reconstruct=dc"]),
    "loop3d_ppmx_char": (cases.field_loop(16, 8), ["mhd.characteristic=true"]),
    "blast3d_wenoz_char_lowmach": (cases.blast(12), ["mhd.reconstruct=wenoz", "mhd.characteristic=true",
                                                     "mhd.low_mach=true"]),
    "blast3d_reflect_lhlld": (cases.blast(12), ["mesh.bc_x1=reflect", "mesh.bc_x2=outflow", "problem.angle=90",
                                                "mhd.rsolver=lhlld", "mhd.lhlld_phi=0.5"]),
    "ot2d_plm_char_dual": (cases.ot(24), ["mhd.reconstruct=plm", "mhd.characteristic=true",
                                          "mhd.dual_energy=true", "mhd.de_eta=0.5"]),
}


def _pair(name, warm=3):
    text, ov = CASES[name]
    ref, mesh = make_pair(text, ov, warm_cycles=warm)
    copy_state(ref, mesh)
    return ref, mesh


@pytest.mark.parametrize("name", sorted(CASES))
def test_fluxes_each_direction(name):
    ref, mesh = _pair(name)
    ndir = 1 + ref.two_d + ref.three_d
    for cur in (0, 1):
        for d in range(ndir):
            ref.fluxes(d, cur)
            mesh.fluxes(d, cur)
            assert_fields(ref, mesh, ("f1", "f2", "f3", "e2x1", "e3x1", "e1x2", "e3x2", "e1x3", "e2x3"),
                          what=f"{name} dir {d} cur {cur}")


@pytest.mark.parametrize("name", sorted(CASES))
def test_fluxes_fused_launch(name):
    ref, mesh = _pair(name)
    ndir = 1 + ref.two_d + ref.three_d
    for d in range(ndir):
        ref.fluxes(d, 1)
    mesh.fluxes_all(1)
    assert_fields(ref, mesh, ("f1", "f2", "f3", "e2x1", "e3x1", "e1x2", "e3x2", "e1x3", "e2x3"), what=name)


@pytest.mark.parametrize("name", sorted(CASES))
def test_corner_emf(name):
    ref, mesh = _pair(name)
    ndir = 1 + ref.two_d + ref.three_d
    for d in range(ndir):
        ref.fluxes(d, 0)
    copy_state(ref, mesh)
    ref.corner_emf()
    mesh.corner_emf()
    assert_fields(ref, mesh, ("e1", "e2", "e3"), what=name)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("out,g0,g1,bdt", [(1, 1.0, 0.0, 3e-3), (1, 0.75, 0.25, 1e-3), (0, 1.0 / 3.0, 2.0 / 3.0, 2e-3)])
def test_update(name, out, g0, g1, bdt):
    ref, mesh = _pair(name)
    ref.update(out, g0, g1, bdt)
    mesh.update(out, g0, g1, bdt)
    assert_fields(ref, mesh, ("u0", "u1", "b1f0", "b2f0", "b3f0", "b1f1", "b2f1", "b3f1"), what=name)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("buf", [0, 1])
def test_boundaries(name, buf):
    ref, mesh = _pair(name)
    ref.boundaries(buf)
    mesh.boundaries(buf)
    assert_fields(ref, mesh, ("u0", "u1", "b1f0", "b2f0", "b3f0", "b1f1", "b2f1", "b3f1"), what=name)


def _split_ient(a):
    return np.delete(a, 5, axis=0), a[5]


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("buf", [0, 1])
def test_cons_to_prim_and_dt(name, buf):
    ref, mesh = _pair(name)
    dref = ref.cons_to_prim(buf, True)
    ddev = mesh.cons_to_prim(buf, True)
    assert abs(ddev - dref) <= 1e-15 * dref, (ddev, dref)
    assert_fields(ref, mesh, ("bcc", "ecc"), what=name)
    dual = any("dual_energy=true" in o for o in CASES[name][1])
    for f in ("w", f"u{buf}"):
        a, b = mesh.get(f), ref.get(f)
        a5, aent = _split_ient(a)
        b5, bent = _split_ient(b)
        if dual:
            assert np.max(np.abs(a - b)) <= 1e-13 * max(1.0, np.max(np.abs(b))), f
        else:
            assert np.array_equal(a5, b5), f
            assert np.max(np.abs(aent - bent)) <= 1e-14 * max(1e-300, np.max(np.abs(bent))), f


@pytest.mark.parametrize("name", sorted(CASES))
def test_fofc_flag_and_repair(name):
    ref, mesh = _pair(name)
    # plant flagged cells: a deterministic scatter of the active cells
    rng = np.random.default_rng(7)
    flag = ref.get("flag")
    act = np.zeros_like(flag, dtype=bool)
    ks, js = (ref.ng if ref.three_d else 0), (ref.ng if ref.two_d else 0)
    act[ks:ref.nk - ks, js:ref.nj - js, ref.ng:ref.ni - ref.ng] = True
    planted = act & (rng.random(flag.shape) < 0.05)
    flag[:] = 0
    flag[planted] = 1
    ref.set("flag", flag)
    mesh.set("flag", flag)
    ndir = 1 + ref.two_d + ref.three_d
    for d in range(ndir):
        ref.fofc_repair(d, 0)
        mesh.fofc_repair(d, 0)
    assert_fields(ref, mesh, ("f1", "f2", "f3", "e2x1", "e3x1", "e1x2", "e3x2", "e1x3", "e2x3"), what=name)
    # the flag test itself, on a state with cells pushed below the floors
    u = ref.get("u1")
    u[0][planted] = -1e-3
    ref.set("u1", u)
    mesh.set("u1", u)
    nr = ref.fofc_flag(1)
    nd = mesh.fofc_flag(1)
    assert nr == nd == int(planted.sum())
    assert_fields(ref, mesh, ("flag",), what=name)


@pytest.mark.parametrize("name", ["blast3d_ppm_hlld", "ot2d_ppm_hlld", "shock1d_plm_hlle", "ot2d_plm_char_dual"])
@pytest.mark.parametrize("bdt", [2e-3, 5e-2])
def test_positivity_limiter(name, bdt):
    ref, mesh = _pair(name)
    ndir = 1 + ref.two_d + ref.three_d
    for d in range(ndir):
        ref.fluxes(d, 0)
    copy_state(ref, mesh)
    for d in range(ndir):
        nr = ref.limit_fluxes(d, bdt)
        nd = mesh.limit_fluxes(d, bdt)
        assert nr == nd, (d, nr, nd)
    assert_fields(ref, mesh, ("f1", "f2", "f3"), tol=1e-14 if "dual" in name else 0.0, what=name)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("fofc", [True, False])
def test_whole_stage(name, fofc):
    text, ov = CASES[name]
    ov = ov + [f"mhd.fofc={'true' if fofc else 'false'}"]
    ref, mesh = make_pair(text, ov, warm_cycles=2)
    copy_state(ref, mesh)
    for (cur, out, g0, g1, bdt) in [(0, 1, 1.0, 0.0, 2e-3), (1, 1, 0.75, 0.25, 5e-4), (1, 0, 1 / 3, 2 / 3, 1.3e-3)]:
        ref.stage(cur, out, g0, g1, bdt)
        mesh.stage(cur, out, g0, g1, bdt)
        assert_fields(ref, mesh, ("u0", "u1", "b1f0", "b2f0", "b3f0", "b1f1", "b2f1", "b3f1"), what=name)
