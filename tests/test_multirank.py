"""The multi-GPU path of bench.py on CPU: one process per rank over gloo (world size 2,
127.0.0.1). Replicas only: the only cross-rank operations are the barrier and the max of the
ranks' device times (no data-path collective); under `--impl reference` rank 0 alone runs the
host baseline and the other ranks exit 0 without output."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    dist = bench.dist_init()
    bench.barrier(dist)
    mx = bench.dist_max(dist, 10.0 + rank)           # slowest rank's time wins
    buf = io.StringIO()
    with redirect_stdout(buf):
        rc = bench.main_reference(type("A", (), {"n": 512, "cpu_n": 8, "warmup": 0, "steps": 1, "gpus": world})(), rank)
    bench.barrier(dist)
    dist.destroy_process_group()
    q.put((rank, mx, rc, buf.getvalue()))


def test_two_ranks_gloo_max_and_reference_gating():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, mx, rc, out = q.get(timeout=300)
        got[r] = (mx, rc, out)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0][0] == got[1][0] == 11.0
    assert got[0][1] == 0 and got[1][1] == 0
    assert got[1][2] == ""                             # rank 1 prints nothing
    assert '"impl": "reference"' in got[0][2]          # rank 0 prints the reference line
