"""Helpers shared by the GPU parity tests: build a reference simulation (the oracle) and a
device mesh from the same input text, copy the full reference state into the device, and
compare fields."""
from __future__ import annotations

import numpy as np

from chasqui_b200 import Mesh, Params, config_from_params, make_config

STATE_FIELDS = ("u0", "u1", "b1f0", "b2f0", "b3f0", "b1f1", "b2f1", "b3f1", "w", "bcc", "ecc",
                "f1", "f2", "f3", "e2x1", "e3x1", "e1x2", "e3x2", "e1x3", "e2x3", "e1", "e2", "e3", "flag")


def make_pair(text: str, overrides=(), precision: str = "fp64", warm_cycles: int = 0):
    from oracle.refsim import RefSim
    ref = RefSim(text, list(overrides))
    if warm_cycles:
        ref.cycles(warm_cycles)
    pin = Params().read_text(text)
    for o in overrides:
        pin.override(o)
    pin.override(f"mhd.precision={precision}")
    mesh = Mesh(make_config(**config_from_params(pin)))
    return ref, mesh


def copy_state(ref, mesh, fields=STATE_FIELDS):
    for f in fields:
        mesh.set(f, ref.get(f))


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| / max(|b|, tiny) over the whole array."""
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


def assert_fields(ref, mesh, fields, tol=0.0, what=""):
    bad = []
    for f in fields:
        a, b = mesh.get(f), ref.get(f)
        e = rel_err(a, b) if tol > 0 else float(np.max(np.abs(a - b)))
        if e > tol:
            idx = np.unravel_index(np.argmax(np.abs(a - b)), a.shape)
            bad.append(f"{f}: err {e:.3e} at {idx} dev={a[idx]!r} ref={b[idx]!r}")
    assert not bad, f"{what}\n" + "\n".join(bad)


def l1_rel(a: np.ndarray, b: np.ndarray) -> float:
    """relative L1 norm sum|a-b| / sum|b| (0 when both are identically zero)."""
    den = float(np.sum(np.abs(b)))
    num = float(np.sum(np.abs(a - b)))
    return num / den if den > 0 else num
