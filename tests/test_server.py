"""Continuous-batching server (chq_server_*): jobs admitted against an HBM budget while
others run, mixed classes on concurrent streams, results identical to the same job run
alone (see solo_history), failures quarantined. Failure injection happens on the host side (a NaN written
into one job's state); nothing here faults or traps the GPU."""
import math

import numpy as np
import pytest

from chasqui_b200 import Batch, ChqError, Mesh, Server, make_config
from chasqui_b200.core import load_library

pytestmark = pytest.mark.gpu


def ot_cfg(n, nlim, **kw):
    return make_config(nx1=n, nx2=n, nx3=1, cfl=0.4, tlim=0.5, nlim=nlim, **kw)


def blast_cfg(n, nlim, **kw):
    return make_config(nx1=n, nx2=n, nx3=n, x1min=-.5, x1max=.5, x2min=-.5, x2max=.5, x3min=-.5, x3max=.5,
                       cfl=0.3, tlim=0.2, nlim=nlim, **kw)


def cpaw_cfg(n, nlim, **kw):
    return make_config(nx1=n, nx2=n, nx3=n, cfl=0.4, tlim=0.6, nlim=nlim, recon=3, **kw)


JOBS = [
    (lambda: ot_cfg(32, 12), "orszag_tang", [-1.0]),
    (lambda: blast_cfg(16, 9), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 7.0]),
    (lambda: ot_cfg(48, 20), "orszag_tang", [2.0]),
    (lambda: cpaw_cfg(16, 8, precision=1), "cpaw", [1, 1, 1, 1.0, 0.1, 1.0, 0.1]),
    (lambda: blast_cfg(12, 5, precision=1), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 9.0]),
    (lambda: ot_cfg(24, 15, recon=3), "orszag_tang", [0.5]),
]


SOLO_CELLS = 1 << 21   # jobs this large run unbatched on their own stream (server default)


def solo_history(cfg, problem, params):
    """The job run by itself: alone on its mesh in the FP64 form (batched FP64 stepping is
    bitwise equal to it), in a batch of its own in the mixed form (the batched FP32 flux
    kernel may fuse multiply-adds differently from the single-mesh one) unless the job is
    large enough for the server to run it unbatched."""
    m = Mesh(cfg)
    m.init_problem(problem, params)
    m.prime(0.0)
    if cfg.precision == 1 and cfg.nx1 * cfg.nx2 * cfg.nx3 < SOLO_CELLS:
        b = Batch([m], graph=True)
        while not b.status()[0]["done"] and (cfg.nlim < 0 or b.status()[0]["cycle"] < cfg.nlim):
            b.cycles(4)
        cyc = b.status()[0]["cycle"]
        b.close()
        return m.history(), cyc
    while (cfg.nlim < 0 or m.clock()["cycle"] < cfg.nlim) and m.clock()["t"] < cfg.tlim:
        m.cycles(4)
    return m.history(), m.clock()["cycle"]


def run_all(srv, max_steps=5000):
    for _ in range(max_steps):
        if srv.step() == 0:
            return
    raise AssertionError("server did not drain")


@pytest.mark.parametrize("autotune", [False, True], ids=["default_settings", "tuned_lanes"])
def test_results_equal_solo_runs_in_any_mix(autotune):
    srv = Server(hbm_budget_bytes=40 << 30, cycles_per_step=3, autotune=autotune)
    ids = [srv.submit(f(), p, prm) for f, p, prm in JOBS]
    run_all(srv)
    for jid, (f, p, prm) in zip(ids, JOBS):
        st = srv.status(jid)
        h, cyc = solo_history(f(), p, prm)
        assert st["state"] == "done", st
        assert st["cycle"] == cyc == f().nlim
        assert np.array_equal(np.array(st["history"]), h), (p, st["history"], h)
        assert st["t_done"] >= st["t_start"] >= st["t_submit"]


@pytest.mark.parametrize("slots", [None, 2])
def test_large_jobs_run_solo_beside_batched_lanes(slots):
    """Jobs of 2^21 cells or more run on their own streams (polled, never waited for) while
    small jobs step in batched lanes; at most `slots` of them at once (default 1: the others
    wait in the queue); every result equals the job run alone."""
    jobs = [
        (lambda: ot_cfg(2048, 4), "orszag_tang", [-1.0]),
        (lambda: blast_cfg(128, 5, precision=1), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 3.0]),
        (lambda: blast_cfg(128, 3), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 4.0]),
        (lambda: blast_cfg(64, 5), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 5.0]),
        (lambda: ot_cfg(32, 12), "orszag_tang", [-1.0]),
        (lambda: blast_cfg(16, 9, precision=1), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 7.0]),
    ]
    srv = Server(hbm_budget_bytes=40 << 30, cycles_per_step=2, solo_slots=slots)
    ids = [srv.submit(f(), p, prm) for f, p, prm in jobs]
    run_all(srv)
    total = 0
    for jid, (f, p, prm) in zip(ids, jobs):
        st = srv.status(jid)
        h, cyc = solo_history(f(), p, prm)
        assert st["state"] == "done", st
        assert st["cycle"] == cyc == f().nlim
        assert np.array_equal(np.array(st["history"]), h), (p, st["history"], h)
        total += f().nlim * f().nx1 * f().nx2 * f().nx3
    s = srv.stats()
    assert s["zone_updates"] == total and s["active"] == 0 and s["used_bytes"] == 0


def test_time_limited_jobs_end_at_their_end_time():
    """Jobs with an end time and no cycle limit. The server sizes their last chunks from the
    mean step so far instead of a cycle count; where that estimate falls short it runs a
    short chunk more. Every job ends on the cycle the job run alone ends on, with its result."""
    box = dict(x1min=-.5, x1max=.5, x2min=-.5, x2max=.5, x3min=-.5, x3max=.5)
    jobs = [
        (lambda: make_config(nx1=32, nx2=32, nx3=1, cfl=0.4, tlim=0.05, nlim=-1), "orszag_tang", [-1.0]),
        (lambda: make_config(nx1=16, nx2=16, nx3=16, cfl=0.3, tlim=0.02, nlim=-1, **box), "blast",
         [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 7.0]),
        (lambda: make_config(nx1=24, nx2=24, nx3=1, cfl=0.4, tlim=0.03, nlim=-1, precision=1), "orszag_tang", [0.5]),
        (lambda: make_config(nx1=1536, nx2=1536, nx3=1, cfl=0.4, tlim=0.002, nlim=-1), "orszag_tang", [-1.0]),
    ]
    srv = Server(hbm_budget_bytes=40 << 30, cycles_per_step=3)
    ids = [srv.submit(f(), p, prm) for f, p, prm in jobs]
    run_all(srv)
    total = 0
    for jid, (f, p, prm) in zip(ids, jobs):
        st = srv.status(jid)
        h, cyc = solo_history(f(), p, prm)
        assert st["state"] == "done", st
        assert st["cycle"] == cyc >= 2 and st["t"] >= f().tlim, (p, st, cyc)
        assert np.array_equal(np.array(st["history"]), h), (p, st["history"], h)
        total += cyc * f().nx1 * f().nx2 * f().nx3
    assert srv.stats()["zone_updates"] == total


def test_jobs_with_diffusion_and_source_terms():
    """Explicit diffusion, cooling and gravity batch with jobs that have the same terms (their
    own coefficients); RKL2 jobs run unbatched. Every result equals the job run alone."""
    jobs = [
        (lambda: ot_cfg(32, 8, nu=2e-3, kappa=2e-3, eta=1e-3), "orszag_tang", [-1.0]),
        (lambda: ot_cfg(24, 9, nu=1e-3), "orszag_tang", [0.5]),
        (lambda: blast_cfg(16, 6, gravity_uniform=1, g1=0.5, g3=-0.25), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 2.0]),
        (lambda: blast_cfg(12, 7, gravity_point=1, gm=0.05, rsoft=0.05), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 3.0]),
        (lambda: ot_cfg(32, 8, cooling=1, lambda0=0.5), "orszag_tang", [-1.0]),
        (lambda: ot_cfg(32, 6, cooling=1, lambda0=0.2, nu=2e-3, gravity_uniform=1, g1=0.3), "orszag_tang", [-1.0]),
        (lambda: ot_cfg(32, 5, eta=0.02, sts=1), "orszag_tang", [-1.0]),
        (lambda: ot_cfg(32, 10), "orszag_tang", [-1.0]),
    ]
    srv = Server(hbm_budget_bytes=40 << 30, cycles_per_step=3)
    ids = [srv.submit(f(), p, prm) for f, p, prm in jobs]
    run_all(srv)
    for jid, (f, p, prm) in zip(ids, jobs):
        st = srv.status(jid)
        h, cyc = solo_history(f(), p, prm)
        assert st["state"] == "done", st
        assert st["cycle"] == cyc == f().nlim
        assert np.array_equal(np.array(st["history"]), h), (p, st["history"], h)


def test_admission_respects_budget_and_drains():
    one = load_library().chq_config_bytes(blast_cfg(16, 6))
    srv = Server(hbm_budget_bytes=int(2.5 * one), cycles_per_step=2)
    ids = [srv.submit(blast_cfg(16, 6), "blast", [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, float(s)]) for s in range(5)]
    seen_queued = False
    for _ in range(2000):
        n = srv.step()
        s = srv.stats()
        assert s["used_bytes"] <= int(2.5 * one)
        assert s["active"] <= 2
        seen_queued |= s["queued"] > 0
        if n == 0:
            break
    assert seen_queued
    assert all(srv.status(j)["state"] == "done" for j in ids)
    assert srv.stats()["zone_updates"] == 5 * 6 * 16 ** 3


def test_rejects_and_quarantines():
    srv = Server(hbm_budget_bytes=1 << 20, cycles_per_step=2)
    with pytest.raises(ChqError):
        srv.submit(ot_cfg(256, 5), "orszag_tang", [-1.0])     # larger than the budget
    srv = Server(hbm_budget_bytes=8 << 30, cycles_per_step=2)
    bad = srv.submit(ot_cfg(32, 10), "orszag_tang", [])      # too few parameters -> FAILED at admission
    good = srv.submit(ot_cfg(32, 10), "orszag_tang", [-1.0])
    victim = srv.submit(ot_cfg(32, 10), "orszag_tang", [-1.0])
    srv.step()
    assert srv.status(bad)["state"] == "failed"
    # inject a NaN into the victim's momentum (host-side failure injection)
    import ctypes as C
    h = srv.job_mesh_handle(victim)
    lib = load_library()
    n = lib.chq_array_size(h, b"u0")
    u = np.empty(n)
    assert lib.chq_download(h, b"u0", u.ctypes.data_as(C.POINTER(C.c_double)), n, None) == 0
    u.reshape(6, -1)[1, 1000:1100] = math.nan
    assert lib.chq_upload(h, b"u0", u.ctypes.data_as(C.POINTER(C.c_double)), n, None) == 0
    run_all(srv)
    assert srv.status(victim)["state"] == "failed"
    assert srv.status(good)["state"] == "done"
    h_solo, _ = solo_history(ot_cfg(32, 10), "orszag_tang", [-1.0])
    assert np.array_equal(np.array(srv.status(good)["history"]), h_solo)
