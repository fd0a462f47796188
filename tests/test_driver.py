"""The command-line driver (chasqui_b200/bin/chasqui, built from chasqui_b200/driver/), a
drop-in for the reference's `chasqui` binary.

CPU: argument and configuration errors, and the host problem generators — every generator of
src/pgen.hpp is run by the driver (`--write-ic`, no GPU) and by the reference's own
Initialize; both initial states go through the reference's Prime and must be bitwise equal.
GPU: whole runs of the driver against the reference binary (oracle/_ref/chasqui) on the same
input: final restart dumps within the cycle-parity tolerance (relative L1 <= 1e-12), history
files within 1e-12, the same output files and end-of-run counters."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from tests import cases

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DRIVER = os.path.join(ROOT, "chasqui_b200", "bin", "chasqui")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "chasqui")

GRESHO = """
[mesh]
nx1 = 24
nx2 = 24
x1min = -0.5
x1max = 0.5
x2min = -0.5
x2max = 0.5
[time]
tlim = 0.1
[problem]
name = gresho
mach = 0.3
"""

UNIFORM = """
[mesh]
nx1 = 12
nx2 = 10
nx3 = 8
[time]
tlim = 0.1
[problem]
name = uniform
dens = 1.3
pres = 0.7
vx = 0.2
vy = -0.1
vz = 0.05
bx = 0.3
by = 0.4
bz = -0.2
"""

PROBLEMS = {
    "orszag_tang": (cases.ot(32), []),
    "blast3d": (cases.blast(12), []),
    "cpaw2d": (cases.cpaw2d(24), []),
    "cpaw1d": (cases.cpaw1d(32), []),
    "field_loop3d": (cases.field_loop(12, 6), []),
    "shock_tube_noise": (cases.shock_tube(64), ["problem.perturb=0.01"]),
    "gresho": (GRESHO, []),
    "uniform3d": (UNIFORM, []),
    "diffusion_b_y": (cases.diffusion("b", 2), ["diffusion.eta=0.02"]),
    "diffusion_temp_x": (cases.diffusion("temp", 1), ["diffusion.kappa=0.003"]),
    "diffusion_v_z": (cases.diffusion("v", 3), ["diffusion.nu=0.02"]),
}


def _write(tmp_path, text, name="in.in"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _run(exe, args, cwd):
    return subprocess.run([exe] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


def read_restart(path):
    with open(path, "rb") as f:
        magic, nx1, nx2, nx3, ng, cycle = struct.unpack("<6i", f.read(24))
        (time,) = struct.unpack("<d", f.read(8))   # offset 24 is already 8-aligned
        (rs,) = struct.unpack("<i", f.read(4))
        f.read(4)
        data = np.frombuffer(f.read(), dtype=np.float64)
    assert magic == 0x43485351 and rs == 8
    return {"nx": (nx1, nx2, nx3), "ng": ng, "cycle": cycle, "time": time, "data": data}


def test_usage_and_configuration_errors(tmp_path):
    r = _run(DRIVER, [], str(tmp_path))
    assert r.returncode == 1 and "usage" in r.stderr
    inp = _write(tmp_path, "[mesh]\nnx1 = 8\n[problem]\nname = blast\n")
    r = _run(DRIVER, ["-i", inp, "mhd.reconstruct=ppm7", "--write-ic", "x.rst"], str(tmp_path))
    assert r.returncode == 1 and "unknown reconstruct" in r.stderr
    r = _run(DRIVER, ["-i", inp, "problem.name=nothing", "--write-ic", "x.rst"], str(tmp_path))
    assert r.returncode == 1 and "unknown problem" in r.stderr
    r = _run(DRIVER, ["-i", inp, "mesh.bc_x1=sticky", "--write-ic", "x.rst"], str(tmp_path))
    assert r.returncode == 1 and "boundary" in r.stderr


@pytest.mark.parametrize("name", sorted(PROBLEMS))
def test_problem_generators_match_reference(name, tmp_path):
    from oracle.refsim import RefSim
    text, ov = PROBLEMS[name]
    inp = _write(tmp_path, text)
    r = _run(DRIVER, ["-i", inp, "--write-ic", "ic.rst"] + ov, str(tmp_path))
    assert r.returncode == 0, r.stderr
    ref = RefSim(text, ov)
    mine = RefSim(text, ov, restart=str(tmp_path / "ic.rst"))
    for f in ("u0", "b1f0", "b2f0", "b3f0", "w", "bcc"):
        a, b = mine.get(f), ref.get(f)
        assert np.array_equal(a, b), (name, f, float(np.max(np.abs(a - b))))
    assert mine.min_dt == ref.min_dt


DRIVER_RUNS = {
    "ot_hst_vtk_rst": (cases.ot(32), ["time.nlim=12", "output.hst_dt=0.01", "output.vtk_dt=0.02",
                                      "output.rst_dt=0.05", "time.ndiag=5"]),
    "blast_fofc_error": (cases.blast(16), ["time.nlim=10", "problem.pres_in=1e4", "problem.pres_out=1e-3",
                                           "time.cfl=0.5", "output.compute_error=true"]),
    "cpaw_tlim_chunks": (cases.cpaw2d(16), ["time.tlim=0.05", "time.ndiag=7"]),
    "diffusion_sts": (cases.diffusion("b", 2), ["diffusion.eta=0.1", "diffusion.sts=true", "time.nlim=8",
                                               "output.hst_dt=0.001"]),
    "limiter_rk2": (cases.ot(24), ["time.integrator=rk2", "mhd.flux_limiter=true", "time.nlim=10",
                                   "output.rst_dt=100"]),
    "gravity_cooling": (cases.ot(24), ["gravity.uniform=true", "gravity.g2=-0.3", "cooling.enabled=true",
                                       "cooling.lambda0=0.2", "time.nlim=10", "output.hst_dt=0.005"]),
    # history alone: rows recorded on the device while cycles run in chunks of replayed graphs
    "blast_hst_chunks": (cases.blast(16), ["time.nlim=40", "problem.pres_in=100", "output.hst_dt=0.009",
                                           "time.ndiag=16"]),
}


def _counters(out):
    keys = ("cycles", "first-order flux corrections applied", "positivity flux limiter activations",
            "super-time-stepping stages \\(total\\)")
    got = {}
    for k in keys:
        m = re.search(r"# " + k + r"\s*[=:]\s*([0-9]+)", out)
        if m:
            got[k] = int(m.group(1))
    return got


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(DRIVER_RUNS))
def test_driver_runs_match_reference_binary(name, tmp_path):
    text, ov = DRIVER_RUNS[name]
    (tmp_path / "ref").mkdir()
    (tmp_path / "dev").mkdir()
    for sub in ("ref", "dev"):
        (tmp_path / sub / "in.in").write_text(text)
    # rst_dt = 1e9 writes only the final dump unless the case sets its own interval
    args = ["-i", "in.in", "output.basename=run", "output.rst_dt=1e9"] + ov
    env = dict(os.environ, OMP_NUM_THREADS="4")
    rr = subprocess.run([REF_BIN] + args, cwd=str(tmp_path / "ref"), capture_output=True, text=True, timeout=900, env=env)
    rd = _run(DRIVER, args, str(tmp_path / "dev"))
    assert rr.returncode == 0, rr.stderr
    assert rd.returncode == 0, rd.stderr
    assert _counters(rd.stdout) == _counters(rr.stdout), (rd.stdout[-600:], rr.stdout[-600:])
    ref_files = sorted(os.listdir(tmp_path / "ref"))
    dev_files = sorted(os.listdir(tmp_path / "dev"))
    assert dev_files == ref_files
    rst = [f for f in ref_files if f.endswith(".rst")]
    assert rst
    for f in rst:
        a, b = read_restart(tmp_path / "dev" / f), read_restart(tmp_path / "ref" / f)
        assert a["cycle"] == b["cycle"] and a["time"] == pytest.approx(b["time"], rel=1e-14, abs=0)
        den = float(np.sum(np.abs(b["data"])))
        assert float(np.sum(np.abs(a["data"] - b["data"]))) <= 1e-12 * den, f
    for f in ref_files:
        if f.endswith(".hst"):
            ha = np.loadtxt(tmp_path / "dev" / f)
            hb = np.loadtxt(tmp_path / "ref" / f)
            assert ha.shape == hb.shape
            np.testing.assert_allclose(ha[:, :10], hb[:, :10], rtol=1e-10, atol=1e-13)
        if f.endswith("_errors.dat"):
            ea = np.loadtxt(tmp_path / "dev" / f)
            eb = np.loadtxt(tmp_path / "ref" / f)
            np.testing.assert_allclose(ea, eb, rtol=1e-9, atol=1e-16)
        if f.endswith(".vtk"):
            va = (tmp_path / "dev" / f).read_bytes()
            vb = (tmp_path / "ref" / f).read_bytes()
            assert len(va) == len(vb)
            # header, time, cycle and coordinates byte for byte; every cell value (built and
            # byte-swapped on the device) to float rounding of the 1e-12 state difference
            cut = vb.index(b"CELL_DATA")
            assert va[:cut] == vb[:cut]
            pa, pb = va[cut:], vb[cut:]
            ncell = int(pb.split(b"\n", 1)[0].split()[1])
            off = len(pb.split(b"\n", 1)[0]) + 1
            for name in (b"rho", b"prs", b"vx1", b"vx2", b"vx3", b"Bx1", b"Bx2", b"Bx3"):
                head = b"SCALARS " + name + b" float\nLOOKUP_TABLE default\n"
                assert pa[off:off + len(head)] == head and pb[off:off + len(head)] == head
                off += len(head)
                fa = np.frombuffer(pa[off:off + 4 * ncell], dtype=">f4")
                fb = np.frombuffer(pb[off:off + 4 * ncell], dtype=">f4")
                np.testing.assert_allclose(fa, fb, rtol=1e-6, atol=1e-7)
                off += 4 * ncell + 1
            assert off == len(pb)
