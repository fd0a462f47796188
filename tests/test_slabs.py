"""Single-job domain decomposition (chasqui_b200/slabs.py) on one GPU: a mesh cut into z slabs
stepped through the slab entry points, with the slabs' halo planes, FOFC flags and reductions
exchanged in-process (LocalExchange), against the same mesh stepped whole. The stage
kernels are the whole mesh's; the decomposition must not change a bit: every cell and face
of the slabs' active planes, the clock, dt and the FOFC count are compared for equality.
Cases cover periodic and outflow z boundaries, 2, 3 and 4 slabs, PPM / PPMX + characteristic
/ WENO-Z, HLLD / LHLLD, FOFC repairs at slab boundaries, explicit diffusion (density minimum
reduced across slabs), point-mass gravity (slab coordinates) and the mixed form."""
import numpy as np
import pytest

from tests.conftest import ROOT  # noqa: F401

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")


def _cfg(n, **kw):
    from chasqui_b200 import make_config
    base = dict(nx1=n, nx2=n, nx3=n, x1min=-0.5, x1max=0.5, x2min=-0.5, x2max=0.5, x3min=-0.5, x3max=0.5,
                recon=2, rsolver=1, integrator=3, cfl=0.4, tlim=10.0, nlim=-1, fofc=1, flatten=1)
    base.update(kw)
    return make_config(**base)


BLAST = ("blast", [10.0, 0.1, 0.12, 1.0, 45.0, 1e-3, 7.0])
STRONG = ("blast", [1e4, 1e-3, 0.12, 1.0, 45.0, 1e-3, 7.0])   # with cfl 0.5: FOFC repairs in most stages
CPAW = ("cpaw", [1.0, 1.0, 1.0, 1.0, 0.1, 1.0, 0.1])


def _whole(cfg, problem, ncyc, via_host=False):
    from chasqui_b200 import Mesh
    m = Mesh(cfg)
    m.init_problem(*problem)
    state0 = {f: m.get(f) for f in FIELDS} if via_host else None
    m.prime(0.0)
    m.cycles(ncyc)
    out = {f: m.get(f) for f in FIELDS}
    ck = m.clock()
    fofc = m.counters()[0]
    ng, nx3 = m.ng, m.nx3
    m.close()
    return out, ck, fofc, ng, nx3, state0


def _slabs(cfg, nslab, problem, ncyc, state0=None):
    import torch
    from chasqui_b200.slabs import LocalExchange, SlabMesh, SlabRun
    stream = torch.cuda.Stream()
    slabs = [SlabMesh(cfg, nslab, r) for r in range(nslab)]
    for s in slabs:
        if state0 is None:
            s.init_problem(*problem)
        else:
            for f in FIELDS:
                s.set_global(f, state0[f])
    run = SlabRun(slabs, LocalExchange(slabs, stream), stream)
    run.prime(0.0)
    run.cycles(ncyc)
    run.synchronize()
    parts = {f: [s.active_planes(f) for s in slabs] for f in FIELDS}
    cks = [s.clock() for s in slabs]
    fofc = [s.counters()[0] for s in slabs]
    launches = sum(s.kernel_launches() for s in slabs)
    for s in slabs:
        s.close()
    return parts, cks, fofc, launches


def _compare(cfg, nslab, problem, ncyc, via_host=False, finite=True):
    whole, ck, fofc, ng, nx3, state0 = _whole(cfg, problem, ncyc, via_host)
    parts, cks, fofcs, launches = _slabs(cfg, nslab, problem, ncyc, state0)
    assert launches > 0
    for f in FIELDS:
        got = np.concatenate(parts[f], axis=-3)
        w = whole[f]
        want = (w if w.ndim == 4 else w[None])[:, ng:ng + nx3]
        want = want if w.ndim == 4 else want[0]
        assert got.shape == want.shape, (f, got.shape, want.shape)
        if finite:
            assert np.all(np.isfinite(want)), f"{f}: the whole mesh broke down; the case proves nothing"
        diff = int(np.count_nonzero(~((got == want) | (np.isnan(got) & np.isnan(want)))))
        assert diff == 0, f"{f}: {diff} values differ between the slabs and the whole mesh"
    for c in cks:
        assert c["cycle"] == ck["cycle"] and c["t"] == ck["t"] and c["dt"] == ck["dt"], (c, ck)
    assert all(x == fofc for x in fofcs), (fofcs, fofc)
    return fofc


@pytest.mark.parametrize("nslab", [2, 3, 4])
def test_blast_periodic_fofc(nslab):
    fofc = _compare(_cfg(24, cfl=0.5), nslab, STRONG, 6)
    assert fofc > 0   # the repairs happen, some of them at slab boundaries


@pytest.mark.parametrize("nslab", [2, 3])
def test_blast_outflow(nslab):
    assert _compare(_cfg(24, bc1=1, bc2=1, bc3=1, cfl=0.5), nslab, STRONG, 6) > 0


def test_blast_reflect_z():
    _compare(_cfg(24, bc3=2), 2, BLAST, 5)


def test_mild_blast_periodic():
    _compare(_cfg(24), 4, BLAST, 6)


def test_cpaw_wenoz_lhlld():
    _compare(_cfg(24, recon=3, rsolver=2, x1min=0.0, x1max=1.0, x2min=0.0, x2max=1.0, x3min=0.0, x3max=1.0,
                  fofc=0), 3, CPAW, 6)


def test_ppmx_characteristic():
    _compare(_cfg(24, recon=4, characteristic=1), 4, BLAST, 5)


def test_explicit_diffusion():
    _compare(_cfg(24, nu=2e-3, eta=2e-3, kappa=1e-3, cfl=0.5), 2, STRONG, 5)


def test_point_mass_gravity():
    _compare(_cfg(24, gravity_point=1, gm=0.05, gx0=0.1, gy0=-0.05, gz0=0.2, rsoft=0.05, cfl=0.5), 3, STRONG, 5)


def test_mixed_form():
    _compare(_cfg(24, precision=1, cfl=0.5), 2, STRONG, 6, finite=False)


def test_initial_state_from_host_slices():
    _compare(_cfg(24), 2, BLAST, 4, via_host=True)


def test_one_slab_is_the_whole_mesh():
    _compare(_cfg(16), 1, BLAST, 4)


def test_slab_rejects_whole_mesh_stepping():
    from chasqui_b200 import ChqError
    from chasqui_b200.slabs import SlabMesh
    s = SlabMesh(_cfg(24), 2, 0)
    with pytest.raises(ChqError):
        s.prime(0.0)
    with pytest.raises(ChqError):
        s.cycles(1)
    s.close()


@pytest.mark.parametrize("integrator", [1, 2, 4])
def test_other_integrators_and_the_limiter(integrator):
    """rk1, rk2 and SSPRK(4,3): other stage tables and output buffers; the positivity limiter
    on (per-slab counts, no exchange needed)"""
    _compare(_cfg(24, integrator=integrator, cfl=0.3 if integrator < 4 else 0.5, flux_limiter=1), 3, STRONG, 5)


def _nccl_single_rank(port, q):
    import os
    import sys
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from chasqui_b200 import set_device
    from chasqui_b200.slabs import DistExchange, SlabMesh, SlabRun
    set_device(0)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        stream = torch.cuda.Stream()
        s = SlabMesh(_cfg(20, cfl=0.5), 1, 0)
        s.init_problem(*STRONG)
        run = SlabRun([s], DistExchange(s, stream), stream)
        run.prime(0.0)
        run.cycles(4)
        run.synchronize()
        q.put(({f: s.get(f) for f in FIELDS}, s.clock(), s.counters()[0]))
        s.close()
    finally:
        dist.destroy_process_group()


def test_dist_exchange_reductions_over_nccl_on_one_rank():
    """DistExchange's FOFC-count sum and dt / density minima as NCCL all-reductions of the
    slab's device step-control words (one rank: no halo messages), against the whole mesh"""
    import socket
    import torch.multiprocessing as mp
    from chasqui_b200 import Mesh
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_single_rank, args=(port, q))
    p.start()
    got, ck, fofc = q.get(timeout=300)
    p.join(timeout=60)
    assert p.exitcode == 0
    m = Mesh(_cfg(20, cfl=0.5))
    m.init_problem(*STRONG)
    m.prime(0.0)
    m.cycles(4)
    for f in FIELDS:
        assert np.array_equal(got[f], m.get(f)), f
    assert ck["t"] == m.clock()["t"] and fofc == m.counters()[0] and fofc > 0
    m.close()
