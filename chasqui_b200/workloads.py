"""Job mixes of the batched-ensemble and serving workloads.

Each job is (chq_config, device problem generator, parameters). Draws come from a seeded
numpy Generator so a mix is reproducible:
  kind      uniform over {Orszag-Tang 2D, CPAW 3D, blast 3D}
  size      OT: N = round(exp(U[ln nmin2, ln nmax2])), N^2 cells;
            3D: N = round(exp(U[ln nmin3, ln nmax3])), N^3 cells
  amplitude U[0.01, 0.2]; plasma beta U[0.1, 10]; scheme PPM or WENO-Z (HLLD, RK3)
Parameter mapping: CPAW amp -> wave amplitude and p = beta * B_par^2 / 2 (B_par = 1);
blast amp -> density-noise amplitude and p_out = beta * b0^2 / 2 (b0 = 1, p_in = 100 p_out);
Orszag-Tang p = beta * B0^2 / 2 (B0 = 1/sqrt(4 pi), amplitude unused).
"""
from __future__ import annotations

import math

import numpy as np

from .core import make_config

KINDS = ("orszag_tang", "cpaw", "blast")


def draw_jobs(n: int, seed: int = 2026, precision: int = 1, nmin2: int = 64, nmax2: int = 1024, nmin3: int = 32,
              nmax3: int = 192, nlim: int = 50, tlim: float = 10.0, t_end=None):
    """n jobs; nlim cycles each (or, with t_end=(lo, hi), an end time U[lo, hi] and no cycle
    limit). Returns a list of dicts with cfg, problem, params, cells, kind."""
    rng = np.random.default_rng(seed)
    jobs = []
    for q in range(n):
        kind = KINDS[int(rng.integers(0, 3))]
        amp = float(rng.uniform(0.01, 0.2))
        beta = float(rng.uniform(0.1, 10.0))
        recon = 2 if rng.random() < 0.5 else 3
        if t_end is not None:
            tl, nl = float(rng.uniform(*t_end)), -1
        else:
            tl, nl = tlim, nlim
        if kind == "orszag_tang":
            N = int(round(math.exp(rng.uniform(math.log(nmin2), math.log(nmax2)))))
            cfg = make_config(nx1=N, nx2=N, nx3=1, recon=recon, cfl=0.4, precision=precision, tlim=tl, nlim=nl)
            params = [beta]
            cells = N * N
        else:
            N = int(round(math.exp(rng.uniform(math.log(nmin3), math.log(nmax3)))))
            if kind == "cpaw":
                cfg = make_config(nx1=N, nx2=N, nx3=N, recon=recon, cfl=0.4, precision=precision, tlim=tl, nlim=nl)
                params = [1.0, 1.0, 1.0, 1.0, beta * 0.5, 1.0, amp]
            else:
                cfg = make_config(nx1=N, nx2=N, nx3=N, x1min=-.5, x1max=.5, x2min=-.5, x2max=.5, x3min=-.5,
                                  x3max=.5, recon=recon, cfl=0.3, precision=precision, tlim=tl, nlim=nl)
                pout = beta * 0.5
                params = [100.0 * pout, pout, 0.1, 1.0, 45.0, amp, float(seed * 1000 + q)]
            cells = N ** 3
        jobs.append({"cfg": cfg, "problem": kind, "params": params, "cells": cells, "kind": kind, "n": N})
    return jobs
