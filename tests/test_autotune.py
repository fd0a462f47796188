"""Flux-kernel autotuning (chq_autotune / chq_set_seglen): the march length changes only the
work decomposition, so results must be bitwise identical for every length; the tuner times
every candidate on the mesh's own state and caches its choice per scheme and shape."""
import numpy as np
import pytest

from chasqui_b200.core import TUNE_LENGTHS
from tests import cases
from tests.parity import copy_state, make_pair

pytestmark = pytest.mark.gpu

FIELDS = ("u0", "b1f0", "b2f0", "b3f0")


@pytest.mark.parametrize("text,ov", [(cases.blast(20), []), (cases.ot(48), ["mhd.reconstruct=wenoz"]),
                                     (cases.field_loop(16, 8), ["mhd.characteristic=true"])],
                         ids=["blast3d_ppm", "ot2d_wenoz", "loop3d_char"])
def test_results_do_not_depend_on_march_length(text, ov):
    out = {}
    for L in (4, 16, 64):
        ref, mesh = make_pair(text, ov)
        copy_state(ref, mesh, FIELDS)
        mesh.seglen = L
        assert mesh.seglen == L
        mesh.prime(0.0)
        mesh.cycles(6)
        out[L] = {f: mesh.get(f) for f in FIELDS}
        ref.close()
    for L in (4, 64):
        for f in FIELDS:
            assert np.array_equal(out[L][f], out[16][f]), (L, f)


def test_autotune_times_every_candidate_and_caches():
    ref, mesh = make_pair(cases.blast(24), ["mhd.reconstruct=ppmx"])
    copy_state(ref, mesh, FIELDS)
    mesh.prime(0.0)
    r = mesh.autotune()
    assert r["seglen"] in TUNE_LENGTHS and mesh.seglen == r["seglen"]
    assert all(t > 0 for t in r["ms"].values())
    assert r["ms"][r["seglen"]] == min(r["ms"].values())
    _, other = make_pair(cases.blast(24), ["mhd.reconstruct=ppmx"])
    r2 = other.autotune()
    assert r2["seglen"] == r["seglen"] and all(t < 0 for t in r2["ms"].values())   # from the cache
    with pytest.raises(Exception):
        mesh.seglen = 0
