"""Flux-kernel autotuning (chq_autotune2 / chq_batch_autotune / chq_set_seglen /
chq_set_xvariant): the march length and the x-sweep variant change only the work
decomposition and the register allocation, so results must be bitwise identical for every
setting; the tuner times every candidate on the mesh's (or the batch's) own state and caches
its choice per scheme, precision and shape (size class for batches)."""
import numpy as np
import pytest

from chasqui_b200 import Batch
from chasqui_b200.core import TUNE_LENGTHS, TUNE_NXVAR
from tests import cases
from tests.parity import copy_state, make_pair

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")


@pytest.mark.parametrize("text,ov", [(cases.blast(20), []), (cases.ot(48), ["mhd.reconstruct=wenoz"]),
                                     (cases.field_loop(16, 8), ["mhd.characteristic=true"])],
                         ids=["blast3d_ppm", "ot2d_wenoz", "loop3d_char"])
def test_results_do_not_depend_on_march_length(text, ov):
    out = {}
    for L, v in ((4, 0), (16, 0), (64, 0), (16, 1)):
        ref, mesh = make_pair(text, ov)
        copy_state(ref, mesh, FIELDS)
        mesh.seglen = L
        mesh.xvariant = v
        assert mesh.seglen == L and mesh.xvariant == v
        mesh.prime(0.0)
        mesh.cycles(6)
        out[(L, v)] = {f: mesh.get(f) for f in FIELDS}
        ref.close()
    for k in ((4, 0), (64, 0), (16, 1)):
        for f in FIELDS:
            assert np.array_equal(out[k][f], out[(16, 0)][f]), (k, f)


def test_mixed_form_tunes_the_march_length_only():
    """the FP32 builds of the two x-sweep variants may round differently, so the tuner leaves
    a mixed-form mesh on variant 0 (its results then do not depend on the tuning)"""
    ref, mesh = make_pair(cases.blast(20), ["mhd.reconstruct=wenoz"], precision="mixed")
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    r = mesh.autotune()
    assert r["xvar"] == 0 and mesh.xvariant == 0
    assert r["xvar_ms"][0] > 0 and all(t < 0 for v, t in r["xvar_ms"].items() if v > 0)
    ref.close()


def test_autotune_times_every_candidate_and_caches():
    ref, mesh = make_pair(cases.blast(24), ["mhd.reconstruct=ppmx"])
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    r = mesh.autotune()
    assert r["seglen"] in TUNE_LENGTHS and mesh.seglen == r["seglen"]
    assert all(t > 0 for t in r["ms"].values())
    assert r["ms"][r["seglen"]] == min(r["ms"].values())
    _, other = make_pair(cases.blast(24), ["mhd.reconstruct=ppmx"])
    assert r["xvar"] in range(TUNE_NXVAR) and mesh.xvariant == r["xvar"]
    assert all(t > 0 for t in r["xvar_ms"].values())
    assert r["xvar_ms"][r["xvar"]] == min(r["xvar_ms"].values())
    r2 = other.autotune()
    assert r2["seglen"] == r["seglen"] and all(t < 0 for t in r2["ms"].values())   # from the cache
    assert r2["xvar"] == r["xvar"] and other.xvariant == r["xvar"]
    with pytest.raises(Exception):
        mesh.seglen = 0
    with pytest.raises(Exception):
        mesh.xvariant = TUNE_NXVAR


def test_batch_autotune_keeps_members_bitwise_equal_to_solo_runs():
    """a tuned batch (its tables rebuilt for every candidate) steps its members exactly as
    each runs alone"""
    specs = [(cases.blast(16), []), (cases.blast(20), []), (cases.ot(40), [])]
    solo, members = [], []
    for text, ov in specs:
        for dst in (solo, members):
            ref, mesh = make_pair(text, ov)
            copy_state(ref, mesh, FIELDS)
            mesh.prime(0.0)
            dst.append(mesh)
            ref.close()
    for m in solo:
        m.cycles(5)
    b = Batch(members, graph=True)
    r = b.autotune()
    assert r["seglen"] in TUNE_LENGTHS and r["xvar"] in range(TUNE_NXVAR)
    assert all(m.seglen == r["seglen"] for m in members)
    b.cycles(5)
    b.status()
    for j, (a, m) in enumerate(zip(solo, members)):
        for f in FIELDS:
            assert np.array_equal(m.get(f), a.get(f)), (j, f)
    b.close()


@pytest.mark.parametrize("text,ov", [(cases.blast(20), []), (cases.ot(48), []),
                                     (cases.blast(16), ["problem.pres_in=1e4", "problem.pres_out=1e-3",
                                                        "time.cfl=0.5"])],
                         ids=["blast3d_ppm", "ot2d_ppm", "blast3d_strong_fofc"])
def test_tma_staging_gives_the_same_bits(text, ov):
    """chq_set_yzvariant(1): the FP64 streaming-PPM march fetches its stencil rows with bulk
    tensor copies instead of per-thread cp.async; same slots, same values, same results"""
    out = {}
    for v, L in ((0, 16), (1, 16), (1, 4), (1, 64)):
        ref, mesh = make_pair(text, ov)
        copy_state(ref, mesh, FIELDS)
        mesh.seglen = L
        mesh.yzvariant = v
        assert mesh.yzvariant == v
        mesh.prime(0.0)
        mesh.cycles(6)
        out[(v, L)] = {f: mesh.get(f) for f in FIELDS}
        ref.close()
    for k in ((1, 16), (1, 4), (1, 64)):
        for f in FIELDS:
            assert np.array_equal(out[k][f], out[(0, 16)][f]), (k, f)


def test_tma_staging_is_tuned_and_limited_to_fp64_ppm():
    ref, mesh = make_pair(cases.blast(24), [])
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    r = mesh.autotune_yz()
    assert r["ms"][0] > 0 and r["ms"][1] > 0
    assert mesh.yzvariant == r["yzvar"] == (1 if r["ms"][1] < r["ms"][0] else 0)
    from chasqui_b200 import ChqError
    for ov, prec in ((["mhd.reconstruct=wenoz"], "fp64"), ([], "mixed"), (["mhd.characteristic=true"], "fp64")):
        _, other = make_pair(cases.blast(16), ov, precision=prec)
        with pytest.raises(ChqError):
            other.yzvariant = 1
        assert other.autotune_yz()["ms"] == {0: -1.0, 1: -1.0}
    ref.close()
