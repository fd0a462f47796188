"""Pins the oracle (the reference built in place against the Kokkos-API shim) to the
reference's own known answers: its bitwise symmetry test, its eigensystem test and the
published CPAW L1 table (README.md:90-96). CPU only."""
import math
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT
from tests import cases

REF = os.path.join(ROOT, "oracle", "_ref")
pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "libchqref.so")),
                                reason="oracle/_ref not built (make -C oracle REF=<reference source tree>)")


def test_reference_symmetry_test_passes():
    r = subprocess.run([os.path.join(REF, "symmetry_test")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert "ALL SYMMETRIC" in r.stdout


def test_reference_eigen_test_passes():
    r = subprocess.run([os.path.join(REF, "eigen_test")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    assert "bad samples = 0" in r.stdout


def cpaw_l1(scheme: str, n: int) -> float:
    """Total L1 error after one period, as compute_error (src/main.cpp:310-327)."""
    from oracle.refsim import RefSim
    s = RefSim(cases.cpaw1d(n), [f"mhd.reconstruct={scheme}", "time.tlim=1.0"])
    u0, b0 = s.get("u0").copy(), s.get("bcc").copy()
    while s.cycles(1000) > 0:
        pass
    assert abs(s.time - 1.0) < 1e-12
    u1, b1 = s.get("u0"), s.get("bcc")
    act = (slice(None), slice(0, 1), slice(0, 1), slice(s.ng, s.ng + n))
    err = np.abs(u1[act] - u0[act]).sum(axis=(1, 2, 3)).tolist() + np.abs(b1[act] - b0[act]).sum(axis=(1, 2, 3)).tolist()
    s.close()
    return sum(e / n for e in err)


# published table (README.md:90-96), HLLD + RK3, CFL 0.4, T = 1
PUBLISHED = {
    "plm": (1.42e-2, 3.99e-3, 9.95e-4),
    "ppm": (1.38e-2, 3.20e-3, 6.65e-4),
    "ppmx": (8.33e-5, 6.25e-6, 5.80e-7),
    "wenoz": (3.93e-5, 4.21e-6, 5.03e-7),
}


@pytest.mark.parametrize("scheme", sorted(PUBLISHED))
def test_cpaw_l1_table(scheme):
    got = [cpaw_l1(scheme, n) for n in (32, 64, 128)]
    pub = PUBLISHED[scheme]
    for g, p in zip(got, pub):
        # the reference source reproduces its own README table to within 6 %
        assert abs(g / p - 1.0) < 0.06, (scheme, got, pub)
    # convergence orders agree with the published ones to 2 significant figures in spirit:
    # |order difference| < 0.15 on each refinement
    for q in range(2):
        og = math.log2(got[q] / got[q + 1])
        op = math.log2(pub[q] / pub[q + 1])
        assert abs(og - op) < 0.15, (scheme, og, op)
