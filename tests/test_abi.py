"""The C ABI boundary without a GPU: libchq.so loads, exports every function that
include/chq.h declares, the ctypes structure matches the C layout, and host-only calls work.
CPU only (no kernel runs)."""
import os
import re
import subprocess
import tempfile

import pytest

from tests.conftest import ROOT, HAVE_GPU

HEADER = os.path.join(ROOT, "include", "chq.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(chq_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    import ctypes
    from chasqui_b200 import core
    lib = ctypes.CDLL(core.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from chasqui_b200 import core
    bound = {n for n, _, _ in core.SIGNATURES}
    assert set(declared_functions()) == bound


def test_no_extra_exports():
    """Only the chq_ C ABI is exported (kernels and helpers stay hidden)."""
    from chasqui_b200 import core
    out = subprocess.run(["nm", "-D", "--defined-only", core.LIB_PATH], capture_output=True, text=True).stdout
    syms = [l.split()[-1] for l in out.splitlines() if " T " in l]
    chq = [s for s in syms if s.startswith("chq_")]
    assert set(chq) == set(declared_functions())


def test_config_struct_layout_matches_c():
    from chasqui_b200 import core
    import ctypes
    fields = [f for f, _ in core.chq_config._fields_]
    src = '#include <stdio.h>\n#include <stddef.h>\n#include "chq.h"\nint main(void){printf("%zu\\n", sizeof(chq_config));'
    for f in fields:
        src += f'printf("%zu\\n", offsetof(chq_config, {f}));'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    assert vals[0] == ctypes.sizeof(core.chq_config)
    for f, off in zip(fields, vals[1:]):
        assert getattr(core.chq_config, f).offset == off, f


def test_config_defaults_are_the_references():
    from chasqui_b200 import default_config
    c = default_config()
    # src/main.cpp:116-142
    assert (c.recon, c.rsolver, c.integrator) == (2, 1, 3)
    assert c.cfl == 0.3 and c.gamma == 5.0 / 3.0
    assert c.dfloor == 1e-10 and c.pfloor == 1e-12 and c.de_eta == 1e-3
    assert c.flatten == 1 and c.fofc == 1 and c.flux_limiter == 0 and c.characteristic == 0
    assert c.lhlld_phi == -1.0 and (c.bc1, c.bc2, c.bc3) == (0, 0, 0)


def test_invalid_configs_are_rejected_without_a_device():
    from chasqui_b200 import Mesh, ChqError, make_config
    for bad in (dict(nx1=0), dict(recon=9), dict(rsolver=5), dict(integrator=7), dict(nx2=1, nx3=4),
                dict(nghost=2, recon=2), dict(bc1=4), dict(precision=3)):
        with pytest.raises(ChqError):
            Mesh(make_config(**bad))


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device error path")
def test_mesh_create_fails_cleanly_without_device():
    from chasqui_b200 import Mesh, ChqError
    with pytest.raises(ChqError):
        Mesh(nx1=8)
