"""Host side of the z-slab decomposition (chasqui_b200/slabs.py) on CPU: slab geometry, the
slicing of whole-mesh arrays, the integer minimum of double bit patterns the reductions rely
on, and DistExchange's ring messages between gloo ranks (world sizes 2 and 3, periodic and
open z) on CPU tensors standing in for the packed halo planes."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def test_slab_planes():
    from chasqui_b200.slabs import slab_planes
    from chasqui_b200 import ChqError
    assert [slab_planes(24, 3, r) for r in range(3)] == [(0, 8), (8, 8), (16, 8)]
    with pytest.raises(ChqError):
        slab_planes(25, 2, 0)
    with pytest.raises(ChqError):
        slab_planes(24, 2, 2)


def test_local_slice_reassembles_the_active_planes():
    from chasqui_b200.slabs import local_slice
    ng, nx3, nslab = 3, 12, 3
    nk = nx3 + 2 * ng
    rng = np.random.default_rng(1)
    cells = rng.random((6, nk, 5, 7))
    faces = rng.random((nk + 1, 6, 8))
    nzl = nx3 // nslab
    got_c, got_f = [], []
    for r in range(nslab):
        koff = r * nzl
        c = local_slice(cells, koff, nzl + 2 * ng, face=False)
        f = local_slice(faces, koff, nzl + 2 * ng, face=True)
        assert c.shape == (6, nzl + 2 * ng, 5, 7) and f.shape == (nzl + 2 * ng + 1, 6, 8)
        # the slab's ghosts are the whole mesh's neighbouring planes
        assert np.array_equal(c[:, :ng], cells[:, koff:koff + ng])
        got_c.append(c[:, ng:ng + nzl])
        got_f.append(f[ng:ng + nzl])
    assert np.array_equal(np.concatenate(got_c, axis=1), cells[:, ng:ng + nx3])
    assert np.array_equal(np.concatenate(got_f, axis=0), faces[ng:ng + nx3])


def test_integer_minimum_of_double_bits_is_the_double_minimum():
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.random(1000) * 10.0 ** rng.integers(-300, 300, 1000), [0.0, np.inf, 5e-324]])
    bits = v.view(np.int64)
    for _ in range(200):
        idx = rng.integers(0, v.size, rng.integers(1, 9))
        assert v[idx].min() == bits[idx].min().view(np.float64)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, periodic, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from chasqui_b200.slabs import DistExchange
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    ex = DistExchange()   # ring messages only (no slab): CPU tensors stand in for halo planes
    n_lo, n_hi = 7, 5     # the downward message is longer (the shared face plane)
    has_lo = periodic or rank > 0
    has_hi = periodic or rank < world - 1
    send_lo = torch.full((n_lo,), 100 * rank + 1, dtype=torch.int64)
    send_hi = torch.full((n_hi,), 100 * rank + 2, dtype=torch.int64)
    recv_lo = torch.full((n_hi,), -1, dtype=torch.int64)
    recv_hi = torch.full((n_lo,), -1, dtype=torch.int64)
    for _ in range(2):   # repeated rounds stay matched
        ex.ring(send_lo, send_hi, recv_lo, recv_hi, has_lo, has_hi)
    nbad = torch.tensor([rank + 1], dtype=torch.int32)
    dist.all_reduce(nbad, op=dist.ReduceOp.SUM)
    mdt = torch.tensor([float(3 + rank)], dtype=torch.float64).view(torch.int64)
    dist.all_reduce(mdt, op=dist.ReduceOp.MIN)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, recv_lo.tolist(), recv_hi.tolist(), int(nbad.item()), float(mdt.view(torch.float64).item())))


@pytest.mark.parametrize("world,periodic", [(2, True), (3, True), (3, False), (2, False)])
def test_ring_exchange_gloo(world, periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, periodic, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, lo, hi, nbad, mdt = q.get(timeout=300)
        got[r] = (lo, hi, nbad, mdt)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        lo, hi, nbad, mdt = got[r]
        lower, upper = (r - 1) % world, (r + 1) % world
        if periodic or r > 0:
            assert lo == [100 * lower + 2] * 5, (r, lo)
        else:
            assert lo == [-1] * 5
        if periodic or r < world - 1:
            assert hi == [100 * upper + 1] * 7, (r, hi)
        else:
            assert hi == [-1] * 7
        assert nbad == world * (world + 1) // 2
        assert mdt == 3.0
