"""Sharding of the ensemble and serving workloads by job (chasqui_b200.dispatch).

On CPU: the assignment is a partition of the draw (disjoint, covering), deterministic, and
balanced (the ranks' totals differ by at most one job's cost); two gloo ranks (127.0.0.1)
compute the same assignment independently and the host-side gather combines their metrics.
On the GPU: two rank processes (sharing one device here; their kernels never wait on each
other) run their shares of a small ensemble, and every job's result equals the result of
the same job run in a single process, bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from chasqui_b200 import dispatch, workloads

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _draw(n=256, **kw):
    return workloads.draw_jobs(n, seed=2026, precision=1, nlim=50, **kw)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shard_jobs_partitions_and_balances(world):
    jobs = _draw()
    costs = [dispatch.job_cost(j) for j in jobs]
    shards = dispatch.shard_jobs(costs, world)
    assert len(shards) == world
    flat = sorted(q for s in shards for q in s)
    assert flat == list(range(len(jobs)))
    loads = [sum(costs[q] for q in s) for s in shards]
    assert max(loads) - min(loads) <= max(costs)
    assert dispatch.shard_jobs(costs, world) == shards


def test_assign_stream_partitions_in_arrival_order():
    jobs = workloads.draw_jobs(500, seed=77, precision=1, t_end=(0.05, 0.5))
    costs = [dispatch.job_cost(j) for j in jobs]
    for world in (1, 2, 4):
        own = dispatch.assign_stream(costs, world)
        assert len(own) == len(jobs) and set(own) <= set(range(world))
        loads = [sum(c for c, o in zip(costs, own) if o == r) for r in range(world)]
        assert max(loads) - min(loads) <= max(costs)
        assert dispatch.assign_stream(costs, world) == own
    assert dispatch.assign_stream(costs, 1) == [0] * len(jobs)


def test_job_cost_counts_zone_updates():
    j = _draw(1)[0]
    assert dispatch.job_cost(j) == j["cells"] * 50
    s = workloads.draw_jobs(1, seed=3, precision=1, t_end=(0.1, 0.1))[0]
    # cells x (cells per dimension) x t_end
    assert dispatch.job_cost(s) == pytest.approx(s["cells"] * s["n"] * 0.1, rel=1e-12)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    from chasqui_b200 import dispatch as dsp, workloads as wl
    dist = bench.dist_init()
    jobs = wl.draw_jobs(64, seed=2026, precision=1, nlim=50)
    mine = dsp.shard_jobs([dsp.job_cost(j) for j in jobs], world)[rank]
    g = dsp.gather(dist, {"jobs_list": mine, "cells_sum": sum(jobs[i]["cells"] for i in mine),
                          "t_max": 1.0 + rank})
    dist.destroy_process_group()
    q.put((rank, mine, g))


def test_two_gloo_ranks_shard_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, mine, g = q.get(timeout=300)
        got[r] = (mine, g)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    jobs = workloads.draw_jobs(64, seed=2026, precision=1, nlim=50)
    a, b = got[0][0], got[1][0]
    assert not set(a) & set(b) and sorted(a + b) == list(range(64))
    for r in (0, 1):
        g = got[r][1]
        assert g["jobs_list"] == a + b                      # rank order, same on both ranks
        assert g["cells_sum"] == sum(j["cells"] for j in jobs)
        assert g["t_max"] == 2.0


def _gpu_rank(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": "0", "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    from chasqui_b200 import Mesh, dispatch as dsp, set_device, workloads as wl
    set_device(0)
    dist = bench.dist_init()
    jobs = wl.draw_jobs(24, seed=2026, precision=1, nlim=10, nmin2=32, nmax2=96, nmin3=24, nmax3=32)
    mine = dsp.shard_jobs([dsp.job_cost(j) for j in jobs], world)[rank]
    res = {}
    for i in mine:
        j = jobs[i]
        m = Mesh(j["cfg"])
        m.init_problem(j["problem"], j["params"])
        m.prime(0.0)
        m.cycles(10)
        res[i] = m.get("u0")
        m.close()
    bench.barrier(dist)
    dist.destroy_process_group()
    q.put((rank, res))


@pytest.mark.gpu
def test_two_ranks_run_their_shares_like_one_process():
    from chasqui_b200 import Mesh, set_device
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, res = q.get(timeout=600)
        got[r] = res
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert not set(got[0]) & set(got[1])
    set_device(0)
    jobs = workloads.draw_jobs(24, seed=2026, precision=1, nlim=10, nmin2=32, nmax2=96, nmin3=24, nmax3=32)
    assert sorted(list(got[0]) + list(got[1])) == list(range(len(jobs)))
    for r in (0, 1):
        for i, u in got[r].items():
            j = jobs[i]
            m = Mesh(j["cfg"])
            m.init_problem(j["problem"], j["params"])
            m.prime(0.0)
            m.cycles(10)
            assert np.array_equal(m.get("u0"), u), (r, i)
            m.close()
