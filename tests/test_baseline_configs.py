"""The benchmark configurations themselves, pinned to the reference at (or near) their own sizes,
plus the device problem generators that build their initial states.

- Orszag-Tang 2D 256^2 (PPM + HLLD + RK3, CFL 0.4, flattening and FOFC on; the reference's
  own generator): 10 cycles and the whole run to t = 0.5, relative L1 <= 1e-12 per field,
  the same clock and the same FOFC count.
- Circularly polarised Alfven wave along 2 pi (1,1,1) on [0,1]^3 (WENO-Z + HLLD + RK3,
  CFL 0.4): the initial state comes from chasqui_b200.ics and reaches the reference through
  its own restart reader (src/restart.hpp:19-56); 10 cycles at 32^3 and 64^3, <= 1e-12.
  One wave period at 32^3, 64^3 and 128^3 against the exact solution (the initial state, as
  the reference's compute_error, src/main.cpp:310-327): the device errors equal the
  reference's at every size (relative 1e-9), so the convergence orders (2.06 and 1.97) equal
  the reference's to two significant figures, second order as README.md:98-99 states.
- Blast 3D with seeded 1e-3 density noise at 128^3 (PPM + HLLD + RK3, FOFC): 10 cycles,
  <= 1e-12, the same FOFC count.
- Device generators (chq_init_problem) against chasqui_b200.ics, the host generator that the
  reference is fed from: the blast bit for bit except the entropy slot (CUDA's pow is within
  2 ulp of the host's), the oblique CPAW and the beta-rescaled Orszag-Tang to
  rounding of the device's sin/cos (relative 1e-13 of each field's maximum).
"""
import math
import os
import tempfile

import numpy as np
import pytest

from chasqui_b200 import Mesh, Params, config_from_params, ics, make_config
from tests import cases
from tests.parity import copy_state, l1_rel, make_pair

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")

CPAW111 = """
[mesh]
nx1 = {n}
nx2 = {n}
nx3 = {n}
[time]
integrator = rk3
cfl = 0.4
tlim = {tlim}
[mhd]
gamma = 1.6666666666666667
reconstruct = wenoz
rsolver = hlld
[problem]
name = cpaw
"""

BLAST_NOISE = """
[mesh]
nx1 = {n}
nx2 = {n}
nx3 = {n}
x1min = -0.5
x1max = 0.5
x2min = -0.5
x2max = 0.5
x3min = -0.5
x3max = 0.5
[time]
integrator = rk3
cfl = 0.3
tlim = 0.2
[mhd]
gamma = 1.6666666666666667
reconstruct = ppm
rsolver = hlld
[problem]
name = blast
"""


def _restart_pair(text, state):
    """reference loaded from a restart file of `state` (ics output), device mesh with the same
    bits (the reference's post-restart boundary fill and con2prim done on both sides)"""
    from oracle.refsim import RefSim
    g, u, b1, b2, b3 = state[:5]
    with tempfile.TemporaryDirectory() as d:
        rst = os.path.join(d, "ic.rst")
        ics.write_restart(rst, g, u, b1, b2, b3)
        ref = RefSim(text, [], restart=rst)
    mesh = Mesh(make_config(**config_from_params(Params().read_text(text))))
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    return ref, mesh


def _ten_cycles(ref, mesh):
    assert mesh.clock()["min_dt"] == pytest.approx(ref.min_dt, rel=1e-15)
    ref.cycles(10)
    mesh.cycles(10)
    ck = mesh.clock()
    assert ck["cycle"] == ref.cycle == 10
    assert ck["t"] == pytest.approx(ref.time, rel=1e-14, abs=0)
    errs = {f: l1_rel(mesh.get(f), ref.get(f)) for f in FIELDS}
    assert max(errs.values()) <= 1e-12, errs
    assert mesh.counters()[0] == ref.fofc_count
    return errs


def test_ot256_ten_cycles():
    ref, mesh = make_pair(cases.ot(256))
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    _ten_cycles(ref, mesh)
    mesh.close()
    ref.close()


def test_ot256_to_tlim():
    """the whole Orszag-Tang run of the benchmark configuration, t = 0 -> 0.5"""
    ref, mesh = make_pair(cases.ot(256))
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    while ref.cycles(1000) > 0:
        pass
    while mesh.clock()["t"] < 0.5:
        mesh.cycles(512)
    ck = mesh.clock()
    assert ref.time == 0.5 and ck["t"] == 0.5
    assert ck["cycle"] == ref.cycle
    errs = {f: l1_rel(mesh.get(f), ref.get(f)) for f in FIELDS}
    assert max(errs.values()) <= 1e-12, errs
    assert mesh.counters()[0] == ref.fofc_count
    mesh.close()
    ref.close()


@pytest.mark.parametrize("n", [32, 64])
def test_cpaw111_ten_cycles(n):
    st = ics.cpaw_oblique(n, (1, 1, 1))
    ref, mesh = _restart_pair(CPAW111.format(n=n, tlim=10.0), st)
    _ten_cycles(ref, mesh)
    mesh.close()
    ref.close()


def _period_l1(sim_cycles, get, n):
    """compute_error of src/main.cpp:310-327: per-cell L1 of u (6) and bcc (3) against the
    initial state, summed over the variables"""
    ng = 3
    act = (slice(None), slice(ng, ng + n), slice(ng, ng + n), slice(ng, ng + n))
    u0, c0 = get("u0").copy(), get("bcc").copy()
    sim_cycles()
    u1, c1 = get("u0"), get("bcc")
    err = np.abs(u1[act] - u0[act]).sum(axis=(1, 2, 3)).tolist() + np.abs(c1[act] - c0[act]).sum(axis=(1, 2, 3)).tolist()
    return sum(e / n ** 3 for e in err)


def test_cpaw111_convergence():
    errs, refs = {}, {}
    for n in (32, 64, 128):
        st = ics.cpaw_oblique(n, (1, 1, 1))
        period = float(st[5])
        ref, mesh = _restart_pair(CPAW111.format(n=n, tlim=repr(period)), st)

        def run_ref():
            while ref.cycles(1000) > 0:
                pass

        def run_dev():
            while mesh.clock()["t"] < period:
                mesh.cycles(256)
        refs[n] = _period_l1(run_ref, ref.get, n)
        errs[n] = _period_l1(run_dev, mesh.get, n)
        assert ref.time == pytest.approx(period, rel=1e-15)
        assert mesh.clock()["t"] == pytest.approx(period, rel=1e-15)
        mesh.close()
        ref.close()
    for n in refs:
        assert errs[n] == pytest.approx(refs[n], rel=1e-9), (n, errs, refs)
    dev = [math.log2(errs[32] / errs[64]), math.log2(errs[64] / errs[128])]
    rfo = [math.log2(refs[32] / refs[64]), math.log2(refs[64] / refs[128])]
    print("cpaw (1,1,1) L1:", errs, "orders device", dev, "reference", rfo)
    assert [float(f"{o:.2g}") for o in dev] == [float(f"{o:.2g}") for o in rfo]
    # the reference's statement for 3D (README.md:98-99): at least second order
    assert min(dev) >= 1.9, (errs, dev)


def test_blast_noise128_ten_cycles():
    st = ics.blast_noise(128)
    ref, mesh = _restart_pair(BLAST_NOISE.format(n=128), st)
    _ten_cycles(ref, mesh)
    mesh.close()
    ref.close()


def _pgen_state(cfg, problem, prm):
    m = Mesh(cfg)
    m.init_problem(problem, prm)
    out = {f: m.get(f) for f in FIELDS}
    m.close()
    return out


def test_device_blast_generator_matches_host():
    """the benchmark's initial state: chq_init_problem('blast') == ics.blast_noise bit for bit
    (density noise, pressure, face fields, momenta, energy), entropy to one ulp of pow"""
    n = 48
    seed = 20261203
    g, u, b1, b2, b3 = ics.blast_noise(n, seed=seed)
    cfg = make_config(nx1=n, nx2=n, nx3=n, x1min=-.5, x1max=.5, x2min=-.5, x2max=.5, x3min=-.5, x3max=.5)
    dev = _pgen_state(cfg, "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, float(seed)])
    for f, a in zip(("b1f0", "b2f0", "b3f0"), (b1, b2, b3)):
        assert np.array_equal(dev[f], a), f
    for c in range(5):
        assert np.array_equal(dev["u0"][c], u[c]), c
    # rho * p / rho^gamma: CUDA's pow is within 2 ulp of the host's, one rounding after it
    s_dev, s_host = dev["u0"][5], u[5]
    assert np.max(np.abs(s_dev - s_host) / np.abs(s_host)) <= 1e-15


@pytest.mark.parametrize("problem", ["cpaw", "orszag_tang"])
def test_device_wave_generators_match_host(problem):
    if problem == "cpaw":
        n = 32
        g, u, b1, b2, b3, _ = ics.cpaw_oblique(n, (1, 1, 1), pres=0.35, amp=0.07)
        cfg = make_config(nx1=n, nx2=n, nx3=n, recon=3)
        dev = _pgen_state(cfg, "cpaw", [1, 1, 1, 1.0, 0.35, 1.0, 0.07])
    else:
        n = 64
        g, u, b1, b2, b3 = ics.orszag_tang(n, beta=2.5)
        cfg = make_config(nx1=n, nx2=n, nx3=1)
        dev = _pgen_state(cfg, "orszag_tang", [2.5])
    for f, a in zip(FIELDS, (u, b1, b2, b3)):
        d = dev[f].reshape(a.shape)
        if f == "u0":
            for c in range(6):
                scale = max(float(np.max(np.abs(a[c]))), 1e-300)
                assert float(np.max(np.abs(d[c] - a[c]))) <= 1e-13 * scale, (f, c)
        else:
            scale = max(float(np.max(np.abs(a))), 1e-300)
            assert float(np.max(np.abs(d - a))) <= 1e-13 * scale, f
