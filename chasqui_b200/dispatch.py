"""Sharding of independent simulation jobs across GPUs (one process per GPU).

The ensemble and serving workloads are sets of independent jobs: no job exchanges data with
another, so they shard by job with no collective on the data path. Every rank sees the same
job list (the same seeded draw or the same request stream) and computes the same assignment
locally; no message decides who runs what. Results and metrics are gathered on the host
afterwards (a gloo or TCP reduction of a few numbers per rank).

  job_cost(job)            work estimate of a job in zone updates: cells x cycles for a job with
                           a cycle limit; for a job with an end time, cells x (cells per
                           dimension) x t_end, proportional to the zone updates of a run whose
                           time step follows the cell size (CFL)
  shard_jobs(costs, world) a whole batch at once: longest job first onto the least-loaded
                           rank (ties: lowest rank), so the ranks' totals differ by at most
                           one job's cost
  assign_stream(costs, world)
                           requests in arrival order: each to the rank with the least work
                           assigned so far (ties: lowest rank); the same on every rank
  gather(dist, local)      sums, maxima and concatenated lists of the ranks' metrics
"""
from __future__ import annotations

import heapq


def job_cost(job: dict) -> float:
    cfg = job["cfg"]
    cells = float(job["cells"])
    if int(cfg.nlim) > 0:
        return cells * float(cfg.nlim)
    dims = 1 + (int(cfg.nx2) > 1) + (int(cfg.nx3) > 1)
    return cells * cells ** (1.0 / dims) * float(cfg.tlim)


def shard_jobs(costs, world: int) -> list[list[int]]:
    """indices of the jobs of each rank (each list in ascending job order)"""
    if world < 1:
        raise ValueError("world size must be at least 1")
    order = sorted(range(len(costs)), key=lambda q: (-float(costs[q]), q))
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for q in order:
        load, r = heapq.heappop(heap)
        out[r].append(q)
        heapq.heappush(heap, (load + float(costs[q]), r))
    return [sorted(s) for s in out]


def assign_stream(costs, world: int) -> list[int]:
    """rank of each request, in arrival order"""
    if world < 1:
        raise ValueError("world size must be at least 1")
    heap = [(0.0, r) for r in range(world)]
    out = []
    for c in costs:
        load, r = heapq.heappop(heap)
        out.append(r)
        heapq.heappush(heap, (load + float(c), r))
    return out


def gather(dist, local: dict) -> dict:
    """Combine the ranks' metrics on the host: keys ending in '_sum' are summed, '_max'
    maximised, '_list' concatenated in rank order; every rank gets the result. With no
    process group (dist None) the local metrics are returned unchanged."""
    if dist is None:
        return dict(local)
    objs = [None] * dist.get_world_size()
    dist.all_gather_object(objs, local)
    out = {}
    for k in local:
        vals = [o[k] for o in objs]
        if k.endswith("_sum"):
            out[k] = sum(vals)
        elif k.endswith("_max"):
            out[k] = max(vals)
        elif k.endswith("_list"):
            out[k] = [x for v in vals for x in v]
        else:
            out[k] = vals
    return out
