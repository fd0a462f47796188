"""The ensemble's job draws on the device.

- A strong blast on a 16^3 mesh puts the r = 0.1 overpressure region in fewer than two cells.
  With WENO-Z the reference's scheme itself breaks down on many such draws (it goes
  non-finite within 50 cycles on about half of them, in FP64): after a FOFC repair in RK
  stages 2 and 3 the reference re-runs the update on a buffer the first update overwrote
  (src/main.cpp:68-91), so a cell driven below the density floor stays there and con2prim's
  floor turns its momentum into velocities of 1e8 and more. The device's FP64 form follows the
  reference bit for bit through such a breakdown (same state the cycle before, non-finite in
  the same cycle). That is why the small-job ensemble draws its 3D meshes from 24^3 up.
- The small-job ensemble of the benchmark (256 jobs, OT 32^2..128^2, CPAW / blast
  24^3..48^3, mixed form, 50 cycles) finishes every job on the batching server.
"""
import os
import tempfile

import numpy as np
import pytest

from chasqui_b200 import Mesh, Params, Server, config_from_params, ics, make_config, workloads
from tests.parity import copy_state, l1_rel

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")

BLAST16 = """
[mesh]
nx1 = 16
nx2 = 16
nx3 = 16
x1min = -0.5
x1max = 0.5
x2min = -0.5
x2max = 0.5
x3min = -0.5
x3max = 0.5
[time]
integrator = rk3
cfl = 0.3
tlim = 10.0
[mhd]
gamma = 1.6666666666666667
reconstruct = wenoz
rsolver = hlld
[problem]
name = blast
"""

# a draw of the small-job distribution (p_in = 100 p_out, p_out = beta / 2) on which the
# reference goes non-finite in cycle 12
AMP, BETA, SEED, FAIL_CYCLE = 0.027384164961978673, 5.457323831627239, 1015, 12


def test_under_resolved_blast_breaks_down_as_in_reference():
    from oracle.refsim import RefSim
    pout = 0.5 * BETA
    g, u, b1, b2, b3 = ics.blast_noise(16, seed=SEED, amp=AMP, pres_in=100.0 * pout, pres_out=pout)
    with tempfile.TemporaryDirectory() as d:
        rst = os.path.join(d, "ic.rst")
        ics.write_restart(rst, g, u, b1, b2, b3)
        ref = RefSim(BLAST16, [], restart=rst)
    mesh = Mesh(make_config(**config_from_params(Params().read_text(BLAST16))))
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    ref.cycles(FAIL_CYCLE - 1)
    mesh.cycles(FAIL_CYCLE - 1)
    for f in FIELDS:
        a, b = mesh.get(f), ref.get(f)
        assert np.isfinite(b).all() and l1_rel(a, b) <= 1e-12, f
    assert mesh.counters()[0] == ref.fofc_count > 0
    ref.cycles(1)
    mesh.cycles(1)
    assert not np.isfinite(ref.get("u0")).all()
    assert not np.isfinite(mesh.get("u0")).all()
    mesh.close()
    ref.close()


def test_small_job_ensemble_finishes_every_job():
    jobs = workloads.draw_jobs(256, seed=2026, precision=1, nlim=50, nmin2=32, nmax2=128, nmin3=24, nmax3=48)
    srv = Server(8 << 30, max_active=100000, cycles_per_step=16)
    ids = [srv.submit(j["cfg"], j["problem"], j["params"]) for j in jobs]
    while srv.step() > 0:
        pass
    st = [srv.status(i) for i in ids]
    srv.close()
    bad = [(q, jobs[q]["kind"], jobs[q]["n"], s["state"]) for q, s in enumerate(st) if s["state"] != "done"]
    assert not bad, bad
