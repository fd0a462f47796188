#!/usr/bin/env python
"""Throughput of the per-Runge-Kutta-stage ideal-MHD path on B200.

A step is one full RK3 cycle (3 stages: fluxes, corner EMF, update + CT, FOFC test and
repair, boundaries, con2prim + dt) over the whole mesh, with dt computed on the device.
Default workload: 3D MHD blast, 512^3, PPM + HLLD + RK3, FOFC and flattening on, seeded
1e-3 density noise, in the FP64 form (headline `value`) and the mixed FP32/FP64 form.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl chasqui|reference] [--n 512]

Multi-GPU: a single mesh does not shard (single-block solver): for the headline N ranks run
N independent replicas ("replicas only"); value = all ranks' zone updates / max-over-ranks
device time. The ensemble and serving workloads shard by job (chasqui_b200.dispatch): every
rank sees the same draw or request stream and runs its share; metrics are gathered on the
host, with no collective on the data path.
Every timing is CUDA-event device time on the mesh's stream. The state (~67 GB FP64 at
512^3) is far larger than L2, so no flush is needed between steps.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s & % HBM peak (FP64 vs mixed); served-jobs p50/p99 latency"
UNIT = "zone-updates/s"
# algorithmic bytes per cell per RK stage (3D, FOFC on); K1 face fluxes alone
BYTES_STEP = {"fp64": 1132, "mixed": 748}
BYTES_K1 = {"fp64": 408, "mixed": 216}


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------------------
def dist_init():
    world = env_int("WORLD_SIZE", 1)
    if world <= 1:
        return None
    import torch.distributed as dist
    import datetime
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return dist


def dist_max(dist, v: float) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def blast_config(n: int, precision: int):
    from chasqui_b200 import make_config
    return make_config(nx1=n, nx2=n, nx3=n, x1min=-0.5, x1max=0.5, x2min=-0.5, x2max=0.5, x3min=-0.5, x3max=0.5,
                       recon=2, rsolver=1, integrator=3, cfl=0.3, fofc=1, flatten=1, precision=precision, tlim=0.2)


BLAST_PARAMS = [10.0, 0.1, 0.1, 1.0, 45.0, 1e-3, 20261203.0]   # p_in, p_out, r, b0, angle, noise, seed


STATE_FIELDS = ("u0", "b1f0", "b2f0", "b3f0")
L1_NAMES = ("rho", "m1", "m2", "m3", "E", "rho_s", "b1f", "b2f", "b3f")


def active_views(st: dict, ng: int = 3):
    """the active cells of u (6 variables) and the active faces of the three face fields"""
    u = st["u0"]
    out = [u[c, ng:-ng, ng:-ng, ng:-ng] for c in range(6)]
    out.append(st["b1f0"][ng:-ng, ng:-ng, ng:-ng - 1 or None])
    out.append(st["b2f0"][ng:-ng, ng:-ng - 1 or None, ng:-ng])
    out.append(st["b3f0"][ng:-ng - 1 or None, ng:-ng, ng:-ng])
    return out


def l1_per_field(a: dict, b: dict) -> tuple[dict, dict]:
    """per conserved variable and face field over the active region: relative L1
    sum|a - b| / sum|b|, and the mean absolute difference per cell (or face)"""
    rel, mean = {}, {}
    for name, x, y in zip(L1_NAMES, active_views(a), active_views(b)):
        den = float(np.sum(np.abs(y), dtype=np.float64))
        num = float(np.sum(np.abs(x - y), dtype=np.float64))
        rel[name] = num / den if den > 0 else num
        mean[name] = num / y.size
    return rel, mean


def run_form(n, precision, steps, warmup, dist, device, sample_clocks=False, profile_cycles=2, keep_state=False,
             pin=None):
    from chasqui_b200 import Mesh
    mesh = Mesh(blast_config(n, precision))
    mesh.init_problem("blast", BLAST_PARAMS)
    mesh.prime(0.0)
    # flux-kernel march length picked by the library's autotuner on this state (the default
    # is 16; the per-length launch times are reported beside the choice). `pin` =
    # (march length, x variant, y/z staging) skips the tuner and sets those, so that a run
    # under a profiler, whose serialised replays distort the tuner's timings, launches the
    # kernels a plain run picked.
    default_len = mesh.seglen
    if pin is not None:
        mesh.seglen, mesh.xvariant, mesh.yzvariant = pin
        tune = {"ms": {}, "seglen": mesh.seglen, "xvar": mesh.xvariant, "default": default_len, "pinned": True,
                "yz": {"yzvar": mesh.yzvariant, "ms": {0: -1.0, 1: -1.0}}}
    else:
        tune = mesh.autotune()
        tune["default"] = default_len
        tune["yz"] = mesh.autotune_yz()   # y/z staging: cp.async (0) or TMA (1), FP64 streaming PPM
    mesh.cycles(warmup)
    mesh.clock()
    l0 = mesh.kernel_launches()
    barrier(dist)
    sampler = ClockSampler(device) if sample_clocks else None
    if sampler:
        sampler.__enter__()
    mesh.record(0)
    mesh.cycles(steps)
    mesh.record(1)
    ms = mesh.elapsed_ms(0, 1)
    if sampler:
        sampler.__exit__()
    launches = mesh.kernel_launches() - l0
    ck = mesh.clock()
    ms_max = dist_max(dist, ms)
    # per-kernel device times (separate short run with per-kernel events)
    mesh.profile(True)
    mesh.cycles(profile_cycles)
    prof = mesh.profile_read(reset=True)
    mesh.profile(False)
    fofc, _ = mesh.counters()
    state = {f: mesh.get(f) for f in STATE_FIELDS} if keep_state else None
    return mesh, {"ms": ms, "ms_max": ms_max, "launches": launches, "clock": ck, "prof": prof,
                  "clocks": sampler.summary() if sampler else None, "fofc": fofc, "tune": tune,
                  "cycles_total": warmup + steps + profile_cycles, "state": state, "t_end": mesh.clock()["t"]}


def config_rates(steps: int = 5, warmup: int = 3) -> dict:
    """zone-updates/s of the other benchmark configurations, timed like the headline (CUDA
    events around whole device cycles, warm-up first): OT 2D 256^2, CPAW 3D 256^3 along
    2 pi (1,1,1) with WENO-Z, and the 512^3 blast with RKL2 diffusion nu = eta = 1e-4 (each
    cycle synchronises once for the RKL2 stage count)."""
    from chasqui_b200 import Mesh, make_config
    out = {}
    runs = [
        ("ot2d_256", dict(nx1=256, nx2=256, nx3=1, cfl=0.4, tlim=0.5), "orszag_tang", [-1.0], (0, 1)),
        ("cpaw3d_256_wenoz", dict(nx1=256, nx2=256, nx3=256, recon=3, cfl=0.4, tlim=10.0), "cpaw",
         [1, 1, 1, 1.0, 0.1, 1.0, 0.1], (0, 1)),
        ("blast3d_512_rkl2", dict(nx1=512, nx2=512, nx3=512, x1min=-.5, x1max=.5, x2min=-.5, x2max=.5, x3min=-.5,
                                  x3max=.5, cfl=0.3, tlim=0.2, nu=1e-4, eta=1e-4, sts=1), "blast", BLAST_PARAMS, (0,)),
    ]
    for name, kw, pg, prm, precs in runs:
        for prec in precs:
            m = Mesh(make_config(precision=prec, **kw))
            m.init_problem(pg, prm)
            m.prime(0.0)
            m.autotune()
            m.cycles(warmup)
            m.clock()
            m.record(0)
            m.cycles(steps)
            m.record(1)
            ms = m.elapsed_ms(0, 1)
            cells = kw["nx1"] * kw["nx2"] * kw["nx3"]
            r = {"value": cells * steps / (ms / 1e3), "ms_per_step": ms / steps, "cells": cells}
            if kw.get("sts"):
                r["rkl2_stages_per_cycle"] = m.sts_stages() / (warmup + steps)
            out[name + ("_mixed" if prec else "_fp64")] = r
            m.close()
    # the decomposed path on one device: the 512^3 blast as two z slabs with in-process halos
    out["blast3d_512_2slabs_one_gpu_fp64"] = slab_run(512, 2, steps, warmup)
    out["ot2d_256_hst_every_cycle_fp64"] = history_rates()
    out["rkl2_batch_64x_ot2d_64_fp64"] = rkl2_batch_rates()
    return out


def slab_run(n: int, nslab: int, steps: int, warmup: int, dist=None, rank: int = 0, local: bool = True) -> dict:
    """The headline blast as z slabs (chasqui_b200/slabs.py): with local=True all nslab slabs
    on this GPU (in-process halo exchange: the cost of the decomposed stage on one device);
    otherwise this rank's slab of nslab ranks with NCCL messages between GPUs. CUDA events on
    the slabs' stream around `steps` cycles; the slowest rank's time."""
    import torch
    from chasqui_b200.slabs import DistExchange, LocalExchange, SlabMesh, SlabRun
    stream = torch.cuda.Stream()
    mine = range(nslab) if local else [rank]
    slabs = [SlabMesh(blast_config(n, 0), nslab, r) for r in mine]
    for s in slabs:
        s.init_problem("blast", BLAST_PARAMS)
    if local:
        ex = LocalExchange(slabs, stream)
    else:
        # the halo planes and step-control words live on the GPUs: an NCCL group beside the
        # gloo group of the timings, created collectively by a first all-reduce
        import datetime
        torch.cuda.set_device(env_int("LOCAL_RANK", 0))
        group = dist.new_group(backend="nccl", timeout=datetime.timedelta(seconds=120))
        dist.all_reduce(torch.zeros(1, device="cuda"), group=group)
        ex = DistExchange(slabs[0], stream, group=group)
    run = SlabRun(slabs, ex, stream)
    run.prime(0.0)
    run.cycles(warmup)
    run.synchronize()
    l0 = sum(s.kernel_launches() for s in slabs)
    barrier(dist)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.cycles(steps)
    e1.record(stream)
    e1.synchronize()
    ms = dist_max(dist, e0.elapsed_time(e1))
    launches = sum(s.kernel_launches() for s in slabs) - l0
    ck = slabs[0].clock()
    fofc = slabs[0].counters()[0]
    for s in slabs:
        s.close()
    return {"value": float(n) ** 3 * steps / (ms / 1e3), "ms_per_step": ms / steps, "slabs": nslab,
            "cycle": ck["cycle"], "fofc_corrections": fofc, "gpu_launches": launches,
            "how": ("all slabs on one GPU, halo planes packed and unpacked in-process" if local else
                    "one slab per rank and GPU, halo planes as NCCL messages to the ring neighbours")}


def rkl2_batch_rates(jobs: int = 64, n: int = 64, cycles: int = 20) -> dict:
    """64 Orszag-Tang 64^2 jobs with RKL2 resistivity (eta from 0.02 to 0.2, so 2 to 5
    super-time-stepping stages per cycle, different per job) stepped as one batch (one host
    read of the stage counts per cycle, then each stage one launch per kernel kind over all
    jobs) against the same jobs one after another through chq_cycles. Host wall clock,
    device synchronised at both ends."""
    from chasqui_b200 import Batch, Mesh, make_config

    def make():
        ms = []
        for q in range(jobs):
            eta = 0.02 + 0.18 * q / (jobs - 1)
            m = Mesh(make_config(nx1=n, nx2=n, nx3=1, cfl=0.4, tlim=1e9, eta=eta, sts=1))
            m.init_problem("orszag_tang", [-1.0])
            m.prime(0.0)
            ms.append(m)
        return ms

    cells = n * n * jobs
    seq = make()
    for m in seq:
        m.cycles(2)
        m.clock()
    t0 = time.perf_counter()
    for m in seq:
        m.cycles(cycles)
    for m in seq:
        m.clock()
    seq_s = time.perf_counter() - t0
    stages = sum(m.sts_stages() for m in seq)
    for m in seq:
        m.close()
    mem = make()
    b = Batch(mem)
    b.cycles(2)
    b.status()
    t0 = time.perf_counter()
    b.cycles(cycles)
    b.status()
    bat_s = time.perf_counter() - t0
    launches = b.kernel_launches()
    b.close()
    for m in mem:
        m.close()
    return {"batched": {"value": cells * cycles / bat_s, "seconds": bat_s},
            "sequential": {"value": cells * cycles / seq_s, "seconds": seq_s},
            "speedup": seq_s / bat_s, "rkl2_stages_per_job_cycle": stages / (jobs * (cycles + 2)),
            "batch_launches_per_cycle": launches / (cycles + 2), "unit": "zone-updates/s",
            "timing": "host wall clock, device synchronised at both ends"}


def history_rates(n: int = 400) -> dict:
    """OT 2D 256^2 with a .hst row after every cycle, both ways the C ABI offers: rows recorded
    on the device (chq_history_record: the sums ride on the end-of-cycle con2prim, the cycles
    stay queued as replayed graphs, one drain at the end) against the per-cycle host output test
    (chq_cycles(1), chq_clock, chq_history: two synchronisations and a separate history pass
    per cycle). Host wall clock from an idle device to the last row on the host."""
    from chasqui_b200 import Mesh, make_config
    kw = dict(nx1=256, nx2=256, nx3=1, cfl=0.4, tlim=1e9)
    cells = 256 * 256
    m = Mesh(make_config(precision=0, **kw))
    m.init_problem("orszag_tang", [-1.0])
    m.prime(0.0)
    m.cycles(5)
    m.clock()
    t0 = time.perf_counter()
    for _ in range(n):
        m.cycles(1)
        m.clock()
        m.history()
    host_s = time.perf_counter() - t0
    m.record_history(1e-12, 0.0, 0.0, capacity=n)
    m.cycles(5)
    m.drain_history(n)
    t0 = time.perf_counter()
    m.cycles(n)
    rows, lost, _ = m.drain_history(n)
    dev_s = time.perf_counter() - t0
    m.record_history(0.0, 0.0, 0.0, capacity=0)
    m.close()
    return {"device_rows": {"value": cells * n / dev_s, "rows": int(len(rows)), "lost": int(lost)},
            "host_rows": {"value": cells * n / host_s, "rows": n},
            "speedup": host_s / dev_s, "cycles": n, "unit": "zone-updates/s",
            "timing": "host wall clock, device idle at both ends"}


def tune_summary(tune):
    """autotuned vs default launch settings of the flux kernel: march length (x variant 0) and
    x-sweep variant (at the best length), ms per launch for each candidate"""
    ms = tune["ms"]
    d = tune.get("default", 16)
    out = {"default_seglen": d, "seglen": tune["seglen"], "flux_ms_per_launch": {str(k): v for k, v in ms.items()},
           "xvar": tune.get("xvar", 0), "flux_ms_per_xvar": {str(k): v for k, v in tune.get("xvar_ms", {}).items()}}
    yz = tune.get("yz")
    if yz:
        out["yz_staging"] = {"chosen": "tma" if yz["yzvar"] == 1 else "cp.async",
                             "flux_ms_per_launch": {"cp.async": yz["ms"][0], "tma": yz["ms"][1]}}
    best = min([t for t in list(ms.values()) + list(tune.get("xvar_ms", {}).values()) +
                (list(yz["ms"].values()) if yz else []) if t > 0], default=-1)
    if ms.get(d, -1) > 0 and best > 0:
        out["speedup_vs_default"] = ms[d] / best
    if tune.get("pinned"):
        out["pinned"] = True
    return out


def e2e_host(mesh, steps, warmup, dist, depth=2):
    """zone-updates/s through the host-buffer C-ABI calls: each step uploads a state from
    pinned host memory, primes it, runs one cycle and downloads the new state
    (chq_run_host_async / chq_run_host_wait). Steps alternate between two meshes with `depth`
    host buffers (jobs in flight) each, so a step's upload overlaps the previous step's cycle
    and download (the link is full duplex and the copy engines are not the SMs); with room for
    one mesh only the steps alternate over its buffers. Device time from the first step's
    start to the last step's end, pipeline fill and drain included."""
    from chasqui_b200 import Mesh, PinnedArray
    mesh.init_problem("blast", BLAST_PARAMS)
    names = ("u0", "b1f0", "b2f0", "b3f0")
    meshes = [mesh]
    try:
        other = Mesh(mesh.cfg)
        meshes.append(other)
    except Exception:
        other = None
    start = [mesh.get(f) for f in names]
    sets = []   # sets[w][b]: host buffers b of mesh w
    for _ in meshes:
        per = []
        for _b in range(depth):
            ps = [PinnedArray(a.shape) for a in start]
            for p, a in zip(ps, start):
                p.array[...] = a
            per.append(ps)
        sets.append(per)
    inflight = [0] * len(meshes)

    def run(q):
        w = q % len(meshes)
        if inflight[w] == depth:
            meshes[w].run_host_wait()
            inflight[w] -= 1
        bufs = sets[w][(q // len(meshes)) % depth]
        meshes[w].run_host_async(*[p.array for p in bufs], 1)
        inflight[w] += 1

    def drain():
        for w, m in enumerate(meshes):
            while inflight[w]:
                m.run_host_wait()
                inflight[w] -= 1

    for q in range(max(4, warmup)):
        run(q)
    drain()
    barrier(dist)
    meshes[0].record(2)
    for q in range(steps):
        run(q)
    for m in meshes:
        m.record(3)   # mesh stream: after the last step's copy into the snapshot area
    drain()
    for m in meshes:
        m.record(4)   # after the downloads (drained)
    ms = max(meshes[0].elapsed_ms_to(2, m, 4) for m in meshes)
    nbytes = sum(a.nbytes for a in start)
    # one job through the blocking call: one upload, `steps` cycles, one download
    arrs = [p.array for p in sets[0][0]]
    mesh.record(5)
    mesh.run_host(*arrs, steps)
    mesh.record(6)
    job_ms = mesh.elapsed_ms(5, 6)
    del sets, arrs
    if other is not None:
        other.close()
    return ms / steps, len(meshes), nbytes, job_ms


def cpu_reference(n: int, warmup: int, max_steps: int, budget_s: float, threads: int):
    """The reference's own kernels (oracle/_ref, OpenMP) on the host cores: blast with
    noise at n^3, timed per cycle."""
    from chasqui_b200 import ics
    from oracle.refsim import RefSim, available
    if not available():
        return None
    g, u, b1, b2, b3 = ics.blast_noise(n)
    text = f"""[mesh]
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
reconstruct = ppm
rsolver = hlld
[problem]
name = blast
"""
    with tempfile.TemporaryDirectory() as d:
        rst = os.path.join(d, "ic.rst")
        ics.write_restart(rst, g, u, b1, b2, b3)
        sim = RefSim(text, [], restart=rst, threads=threads)
    for _ in range(warmup):
        sim.cycles(1)
    times = []
    t_start = time.perf_counter()
    while len(times) < max_steps:
        t0 = time.perf_counter()
        sim.cycles(1)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s and len(times) >= 1:
            break
    sim.close()
    return times


def _job_ok(m, cycles: int) -> bool:
    """a job finished: its clock ran all cycles and its history sums are finite"""
    return m.clock()["cycle"] == cycles and bool(np.isfinite(m.history()).all())


def ensemble(njobs: int, cycles: int, seed: int, cps: int, sizes=(64, 1024, 32, 192), dist=None, rank: int = 0,
             world: int = 1) -> dict:
    """The ensemble configuration: njobs seeded jobs (OT 2D sizes[0]^2..sizes[1]^2, CPAW /
    blast 3D sizes[2]^3..sizes[3]^3, PPM or WENO-Z, mixed precision), `cycles` cycles each:
    all submitted at once to the batching server vs the same jobs as sequential one-job runs
    and vs every job on its own stream at once. Every arm checks each job (all cycles run,
    finite state); the rates count the zone updates of the jobs that finished in that arm.
    With several ranks every rank draws the same jobs and runs its share (dispatch.shard_jobs);
    each arm starts at a barrier, its time is the slowest rank's and its zone updates the
    sum over ranks."""
    from chasqui_b200 import Mesh, Server, dispatch, workloads
    drawn = workloads.draw_jobs(njobs, seed=seed, precision=1, nlim=cycles, nmin2=sizes[0], nmax2=sizes[1],
                                nmin3=sizes[2], nmax3=sizes[3])
    mine = dispatch.shard_jobs([dispatch.job_cost(j) for j in drawn], world)[rank]
    jobs = [drawn[q] for q in mine]
    zu_all = sum(j["cells"] for j in drawn) * cycles

    def server_arm(autotune, subset=None):
        barrier(dist)
        srv = Server(150 << 30, max_active=100000, cycles_per_step=cps, autotune=autotune)
        t0 = time.perf_counter()
        ids = [srv.submit(j["cfg"], j["problem"], j["params"]) for j in (jobs if subset is None else subset)]
        steps = 0
        while srv.step() > 0:
            steps += 1
        t = time.perf_counter() - t0
        done = [srv.status(i)["state"] == "done" for i in ids]
        srv.close()
        return t, steps, done

    # untimed warm-up with default settings on the 16 smallest jobs (kernel loading and first
    # allocations, outside every arm; the autotuner's cache stays empty)
    server_arm(False, sorted(jobs, key=lambda j: j["cells"])[:16])
    # the server with its default launch settings, then with every lane's batch tuned by the
    # library's autotuner (first tuning of each lane inside the timed region)
    t_batched, steps, done_b = server_arm(False)
    t_tuned, _, done_t = server_arm(True)
    done_s = []
    barrier(dist)
    t0 = time.perf_counter()
    for j in jobs:
        m = Mesh(j["cfg"])
        m.init_problem(j["problem"], j["params"])
        m.prime(0.0)
        m.cycles(cycles)
        done_s.append(_job_ok(m, cycles))
        m.close()
    t_seq = time.perf_counter() - t0
    # every job on its own mesh stream at once (no batching, no server)
    barrier(dist)
    t0 = time.perf_counter()
    meshes = []
    for j in jobs:
        m = Mesh(j["cfg"])
        m.init_problem(j["problem"], j["params"])
        m.prime(0.0)
        meshes.append(m)
    for m in meshes:
        m.cycles(cycles)
    for m in meshes:
        m.clock()
    t_con = time.perf_counter() - t0
    done_c = [_job_ok(m, cycles) for m in meshes]
    for m in meshes:
        m.close()

    def zu(done):
        return sum(j["cells"] for j, d in zip(jobs, done) if d) * cycles

    g = dispatch.gather(dist, {
        "done_b_sum": sum(done_b), "done_s_sum": sum(done_s), "done_c_sum": sum(done_c), "done_t_sum": sum(done_t),
        "zu_b_sum": zu(done_b), "zu_s_sum": zu(done_s), "zu_c_sum": zu(done_c), "zu_t_sum": zu(done_t),
        "t_b_max": t_batched, "t_s_max": t_seq, "t_c_max": t_con, "t_t_max": t_tuned, "steps_max": steps,
        "jobs_list": [len(jobs)]})
    out = {"jobs": len(drawn), "cycles_each": cycles, "zone_updates": zu_all, "sizes": list(sizes),
           "done": {"batched": g["done_b_sum"], "sequential": g["done_s_sum"], "concurrent_streams": g["done_c_sum"],
                    "batched_autotuned": g["done_t_sum"]},
           "batched": {"seconds": g["t_b_max"], "value": g["zu_b_sum"] / g["t_b_max"], "server_steps": g["steps_max"],
                       "tiles": "the members' default launch settings (the server's default)"},
           "batched_autotuned": {"seconds": g["t_t_max"], "value": g["zu_t_sum"] / g["t_t_max"],
                                 "tiles": "autotuned per lane (march length, x-sweep variant), timing included"},
           "autotuned_vs_default": g["t_b_max"] / g["t_t_max"],
           "sequential": {"seconds": g["t_s_max"], "value": g["zu_s_sum"] / g["t_s_max"]},
           "concurrent_streams": {"seconds": g["t_c_max"], "value": g["zu_c_sum"] / g["t_c_max"]},
           "speedup_batched_vs_sequential": g["t_s_max"] / g["t_b_max"],
           "timing": "host wall clock around submit-to-drain, device synchronised at the end"}
    if world > 1:
        out["sharding"] = {"ranks": world, "jobs_per_rank": g["jobs_list"],
                           "how": "same seeded draw on every rank, longest job first onto the least-loaded rank"}
    out["all_done"] = min(out["done"].values()) == len(drawn)
    if not out["all_done"]:
        print(f"ensemble: jobs that did not finish: {out['done']} of {len(drawn)}", file=sys.stderr)
    return out


def run_alone(job) -> tuple[float, int, bool]:
    """One request run by itself through the public Mesh API (create, generate, prime, cycles
    to its end time, history, close): host wall seconds, zone updates, finished with a
    finite state."""
    from chasqui_b200 import Mesh
    t0 = time.perf_counter()
    m = Mesh(job["cfg"])
    m.init_problem(job["problem"], job["params"])
    m.prime(0.0)
    tl, nl = float(job["cfg"].tlim), int(job["cfg"].nlim)
    while True:
        ck = m.clock()
        if not ck["t"] < tl or (nl >= 0 and ck["cycle"] >= nl):
            break
        m.cycles(32)
    ok = bool(np.isfinite(m.history()).all())
    m.close()
    return time.perf_counter() - t0, int(ck["cycle"]) * int(job["cells"]), ok


_ALONE: dict = {}


def fifo_one_at_a_time(service, arrivals) -> tuple[np.ndarray, float]:
    """Completion times of a first-in first-out queue with one job on the device at a time:
    each request starts when it has arrived and the previous one has finished, and takes its
    measured service time. Returns the latencies and the last completion time."""
    done = 0.0
    lat = []
    for s, a in zip(service, arrivals):
        done = max(done, a) + s
        lat.append(done - a)
    return np.array(lat), done


def serving(njobs: int, rate: float, precision: int, seed: int, t_end=(0.005, 0.05), nmax2=512, nmax3=96,
            cps=4, dist=None, rank: int = 0, world: int = 1, one_at_a_time: bool = False) -> dict:
    """The serving configuration, scaled: njobs requests with Poisson arrivals at `rate` jobs/s,
    kinds and sizes from the ensemble distribution (capped at nmax2^2 / nmax3^3), end time
    U[t_end]; submitted to the server as they arrive; time-to-solution per job. With several
    ranks every rank sees the same request stream and serves the requests that
    dispatch.assign_stream gives it (least assigned work so far); latencies are pooled and
    the throughput is all ranks' zone updates over the slowest rank's wall time.
    one_at_a_time: also the same requests served one job at a time (each request run alone,
    its service time measured, completions from a first-in first-out queue over the same
    arrival times; fifo_one_at_a_time)."""
    from chasqui_b200 import Server, dispatch, workloads
    drawn = workloads.draw_jobs(njobs, seed=seed, precision=precision, nmax2=nmax2, nmax3=nmax3, t_end=t_end)
    rng = np.random.default_rng(seed + 1)
    arr_all = np.cumsum(rng.exponential(1.0 / rate, njobs))
    owner = dispatch.assign_stream([dispatch.job_cost(j) for j in drawn], world)
    jobs = [j for j, o in zip(drawn, owner) if o == rank]
    arrivals = np.array([a for a, o in zip(arr_all, owner) if o == rank])
    njobs = len(jobs)
    barrier(dist)
    srv = Server(150 << 30, max_active=100000, cycles_per_step=cps)
    ids = []
    nxt = 0
    base = srv.stats()["clock"]
    while True:
        now = srv.stats()["clock"] - base
        while nxt < njobs and arrivals[nxt] <= now:
            j = jobs[nxt]
            ids.append(srv.submit(j["cfg"], j["problem"], j["params"]))
            nxt += 1
        busy = srv.step()
        if busy == 0:
            if nxt >= njobs:
                break
            time.sleep(max(0.0, min(0.01, arrivals[nxt] - (srv.stats()["clock"] - base))))
    st = [srv.status(i) for i in ids]
    srv.close()
    g = dispatch.gather(dist, {
        "lat_list": [s["t_done"] - s["t_submit"] for s in st],
        "zu_sum": sum(s["zone_updates"] for s in st),
        "wall_max": (max(s["t_done"] for s in st) - base) if st else 0.0,
        "done_sum": sum(s["state"] == "done" for s in st)})
    lat = np.array(g["lat_list"])
    out = {"requests": len(drawn), "rate_jobs_per_s": rate, "precision": "mixed" if precision else "fp64",
           "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
           "zone_updates_per_s": g["zu_sum"] / g["wall_max"], "done": g["done_sum"],
           "t_end": list(t_end), "max_n2d": nmax2, "max_n3d": nmax3}
    if world > 1:
        out["sharding"] = {"ranks": world, "how": "same request stream on every rank, each request to the "
                                                  "rank with the least assigned work"}
    if one_at_a_time:
        # service times do not depend on the arrival rate: measured once per request set
        key = (precision, seed, tuple(t_end), nmax2, nmax3, len(drawn), rank, world)
        if key not in _ALONE:
            _ALONE[key] = [run_alone(j) for j in jobs]
        runs = _ALONE[key]
        lat1, last = fifo_one_at_a_time([r[0] for r in runs], arrivals)
        g1 = dispatch.gather(dist, {"lat_list": lat1.tolist(), "zu_sum": sum(r[1] for r in runs),
                                    "wall_max": last, "done_sum": sum(r[2] for r in runs)})
        l1 = np.array(g1["lat_list"])
        out["one_at_a_time"] = {"p50_s": float(np.percentile(l1, 50)), "p99_s": float(np.percentile(l1, 99)),
                                "zone_updates_per_s": g1["zu_sum"] / g1["wall_max"], "done": g1["done_sum"],
                                "how": "each request run alone (measured), first-in first-out over the same "
                                       "arrival times"}
        out["server_vs_one_at_a_time"] = {"throughput": out["zone_updates_per_s"] / out["one_at_a_time"]["zone_updates_per_s"],
                                          "p50": out["one_at_a_time"]["p50_s"] / out["p50_s"],
                                          "p99": out["one_at_a_time"]["p99_s"] / out["p99_s"]}
    return out


def serving_study(args, dist, rank, world) -> dict:
    """The serving configuration at its own size range: kinds and sizes of the ensemble draw
    (64^2..1024^2, 32^3..192^3), t_end U[0.05, 0.5], Poisson arrivals, the 150 GB budget, for
    the mixed and FP64 forms, with the one-job-at-a-time arm. Requests per leg: --srv-jobs."""
    out = []
    for prec in (1, 0):
        for r in args.srv_rates.split(","):
            out.append(serving(args.srv_jobs, float(r), prec, 77, t_end=(0.05, 0.5), nmax2=1024, nmax3=192, cps=8,
                               dist=dist, rank=rank, world=world, one_at_a_time=True))
            if rank == 0:   # each leg as it completes (a long study may be cut short)
                print(json.dumps({"serving_leg": out[-1]}), file=sys.stderr, flush=True)
    return {"serving_study": out}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# --------------------------------------------------------------------------------------
def workload_config(n: int, world: int, sample_of: int | None = None) -> dict:
    """The `config` of an arm: the workload it times. `sample_of`: the size of the workload the
    timed mesh is a bounded sample of (the reference arm, whose host state at 512^3 the sample
    budget does not allow)."""
    gb = 67.0 * (n / 512.0) ** 3   # FP64 state, ~67 GB at 512^3
    c = {"workload": f"blast3d {n}^3 ppm+hlld+rk3 fofc flatten, seeded 1e-3 density noise, FP64 form",
         "cells": int(n) ** 3, "parallelism": "replicas" if world > 1 else "single",
         "l2": f"state (~{gb:.0f} GB) >> L2; no flush needed"}
    if sample_of is not None and sample_of != n:
        c["sample_of"] = f"blast3d {sample_of}^3 (same problem, same per-cell work; rate per zone update)"
    return c


def main_reference(args, rank):
    if rank != 0:
        return 0
    threads = host_threads()
    n = args.cpu_n
    times = cpu_reference(n, args.warmup, args.steps, 1e9, threads)
    if times is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle REF=<reference source tree>)"}))
        return 0
    per = statistics.mean(times)
    v = n ** 3 / per
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(n, args.gpus, sample_of=args.n),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"blast3d {n}^3 with 1e-3 noise (a bounded sample of the {args.n}^3 workload: "
                                   f"the same problem at the largest size whose host run fits the sample "
                                   f"budget), {len(times)} RK3 cycles after {args.warmup} warm-up; reference "
                                   f"kernels, OpenMP dispatch"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="chasqui", choices=["chasqui", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--cpu-n", type=int, default=256)
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ens-jobs", type=int, default=256)
    ap.add_argument("--ens-cycles", type=int, default=50)
    ap.add_argument("--srv-jobs", type=int, default=120)
    ap.add_argument("--srv-rates", default="10,40")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--serving-study", action="store_true",
                    help="only the serving configuration at its own size range (see serving_study)")
    ap.add_argument("--flux-settings", default=None, metavar="SEGLEN,XVAR,YZ",
                    help="set the FP64 headline's flux launch settings (march length, x variant, y/z "
                         "staging 0 = cp.async / 1 = TMA) instead of autotuning them")
    ap.add_argument("--slabs", action="store_true",
                    help="only the headline blast decomposed into one z slab per rank (strong scaling)")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)
    rank, local = env_int("RANK", 0), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return main_reference(args, rank)

    from chasqui_b200 import set_device
    dist = dist_init()
    world = env_int("WORLD_SIZE", 1)
    set_device(local)
    if args.slabs:
        r = slab_run(args.n, world, args.steps, args.warmup, dist, rank, local=False)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
                              "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic", "config": dict(workload_config(args.n, world), parallelism=f"z slabs x{world}"),
                              "slabs": r}))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    if args.serving_study:
        res = serving_study(args, dist, rank, world)
        if rank == 0:
            print(json.dumps(res))
        if dist is not None:
            dist.destroy_process_group()
        return 0
    n = args.n
    hbm, peak_kind = peaks()

    pin = tuple(int(v) for v in args.flux_settings.split(",")) if args.flux_settings else None
    if pin is not None and len(pin) != 3:
        raise SystemExit("--flux-settings wants SEGLEN,XVAR,YZ")
    mesh, r64 = run_form(n, 0, args.steps, args.warmup, dist, local, sample_clocks=True,
                         keep_state=not args.no_mixed, pin=pin)
    zones = float(n) ** 3
    value = world * zones * args.steps / (r64["ms_max"] / 1e3)
    ms_step = r64["ms_max"] / args.steps
    prof = r64["prof"]
    k1_ms, k1_n = prof["fluxes"]
    k1_avg_s = (k1_ms / max(k1_n, 1)) / 1e3
    k1_gbs = BYTES_K1["fp64"] * zones / k1_avg_s / 1e9
    step_gbs = (zones * args.steps / (r64["ms"] / 1e3)) * 3 * BYTES_STEP["fp64"] / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            bpc = json.load(f).get("fluxes_fp64_bytes_per_cell")
        if bpc:
            traffic = bpc * zones   # ncu DRAM bytes of one K1 launch at 128^3, scaled by cells
    e2e = None
    if not args.no_e2e:
        # jobs in flight per mesh (each holds its own 10 GB of pinned host state); one when
        # several ranks share the host's memory
        per, nmesh, nbytes, job_ms = e2e_host(mesh, args.steps, args.warmup, dist, depth=2 if world == 1 else 1)
        per = dist_max(dist, per)
        job = dist_max(dist, job_ms)
        e2e = {"value": world * zones / (per / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes, "ms_per_step": per,
               "call": "chq_run_host_async + chq_run_host_wait (pinned host state -> prime -> 1 cycle -> host "
                       f"state), steps alternating over {nmesh} mesh(es)",
               "job": {"value": world * zones * args.steps / (job / 1e3), "cycles_per_call": args.steps,
                       "h2d_bytes": nbytes, "d2h_bytes": nbytes}}
    mesh.close()
    del mesh

    mixed = None
    if not args.no_mixed:
        meshm, rm = run_form(n, 1, args.steps, args.warmup, dist, local, keep_state=True)
        vm = world * zones * args.steps / (rm["ms_max"] / 1e3)
        l1, l1_abs = l1_per_field(rm["state"], r64["state"])
        rm["state"] = r64["state"] = None
        pm = rm["prof"]
        km, kn = pm["fluxes"]
        mixed = {"value": vm, "ms_per_step": rm["ms_max"] / args.steps,
                 "hbm_frac_step": (zones * args.steps / (rm["ms"] / 1e3)) * 3 * BYTES_STEP["mixed"] / 1e9 / hbm,
                 "k1_gbs": BYTES_K1["mixed"] * zones / ((km / max(kn, 1)) / 1e3) / 1e9,
                 "speedup_vs_fp64": vm / value,
                 "kernel_ms_per_step": {k: v[0] / 2 for k, v in pm.items()},
                 "autotune": tune_summary(rm["tune"]),
                 "l1_vs_fp64": {"per_field": l1, "max": max(l1.values()), "mean_abs_per_cell": l1_abs,
                                "cycles": rm["cycles_total"],
                                "t_fp64": r64["t_end"], "t_mixed": rm["t_end"],
                                "what": "relative L1 sum|mixed - fp64| / sum|fp64| and mean |mixed - fp64| "
                                        "over the active cells (u) and faces (b?f) after the same number of "
                                        "cycles from the same initial state (b3f starts at zero, so its "
                                        "relative figure is against a small norm)"}}
        meshm.close()
        del meshm

    cfgs = None
    if rank == 0 and not args.no_configs and n == 512:
        cfgs = config_rates()

    ens = None
    if not args.no_ensemble:
        ens = ensemble(args.ens_jobs, args.ens_cycles, 2026, 16, dist=dist, rank=rank, world=world)
        # the same draw restricted to small meshes (32^2..128^2, 24^3..48^3), where one job
        # alone cannot fill the device and batching is what keeps it busy. (Below 24^3 the
        # blast's r = 0.1 region covers fewer than two cells and the scheme itself breaks down
        # on many strong-blast WENO-Z draws, in FP64 as in the reference.)
        ens["small_jobs"] = ensemble(args.ens_jobs, args.ens_cycles, 2026, 16, sizes=(32, 128, 24, 48), dist=dist,
                                     rank=rank, world=world)
    srv = None
    if not args.no_serving:
        srv = [serving(args.srv_jobs, float(r), prec, 77, dist=dist, rank=rank, world=world, one_at_a_time=True)
               for r in args.srv_rates.split(",") for prec in (1, 0)]
        # the device saturated by small jobs (a burst of requests that one job alone cannot
        # keep the device busy with): continuous batching against one job at a time
        for prec in (1, 0):
            leg = serving(300, 1000.0, prec, 78, nmax2=128, nmax3=48, dist=dist, rank=rank, world=world,
                          one_at_a_time=True)
            leg["leg"] = "burst: 300 requests at 1000 jobs/s, 64^2-128^2 and 32^3-48^3, t_end U[0.005, 0.05]"
            srv.append(leg)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = host_threads()
        times = cpu_reference(args.cpu_n, 1, 20, 20.0, threads)
        if times:
            cpu = {"value": args.cpu_n ** 3 / statistics.mean(times), "unit": UNIT, "cores": threads,
                   "kind": "reference",
                   "sample": f"blast3d {args.cpu_n}^3 with 1e-3 noise, {len(times)} RK3 cycles, OpenMP on all host threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(n, world),
            "hbm_frac_step": step_gbs / hbm,
            "roofline": {"bound": "hbm", "achieved": k1_gbs, "peak": hbm, "unit": "GB/s", "frac": k1_gbs / hbm,
                         "traffic": traffic, "kernel": "flux_yz_kernel + flux_x_kernel (K1, all 3 directions, per stage)",
                         "peak_kind": peak_kind, "bytes_per_cell": BYTES_K1["fp64"]},
            "kernel_ms_per_step": {k: v[0] / 2 for k, v in prof.items()},
            "gpu_launches": r64["launches"],
            "clocks": r64["clocks"],
            "fofc_corrections": r64["fofc"],
            "autotune": tune_summary(r64["tune"]),
            "e2e": e2e,
            "mixed": mixed,
            "configs": cfgs,
            "ensemble": ens,
            "serving": srv,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
