"""Parameter semantics of the drop-in (src/params.hpp:17-92, src/main.cpp:113-185). CPU only."""
import pytest

from chasqui_b200.params import Params, ParamError, config_from_params

TEXT = """
# comment line
[mesh]
nx1 = 64   # trailing comment
nx2=32
 x1min =  -0.5
[mhd]
reconstruct = wenoz
fofc = no
flatten = YES
[problem]
name = orszag_tang
"""


def test_reader_blocks_comments_whitespace():
    p = Params().read_text(TEXT)
    assert p.get_int("mesh", "nx1") == 64
    assert p.get_int("mesh", "nx2") == 32
    assert p.get_real("mesh", "x1min") == -0.5
    assert p.get_string("problem", "name") == "orszag_tang"


def test_overrides_win_and_defaults_are_recorded():
    p = Params().read_text(TEXT)
    p.override("mesh.nx1=128")
    p.override(" time.cfl = 0.4 ")
    assert p.get_int("mesh", "nx1") == 128
    assert p.get_or_add_real("time", "cfl", 0.3) == 0.4
    assert p.get_or_add_int("time", "nlim", -1) == -1
    assert p.has("time", "nlim")
    with pytest.raises(ParamError):
        p.override("no_equals_sign")
    with pytest.raises(ParamError):
        p.get_string("nope", "missing")


def test_bool_spellings():
    p = Params().read_text(TEXT)
    assert p.get_or_add_bool("mhd", "fofc", True) is False
    assert p.get_or_add_bool("mhd", "flatten", False) is True
    assert p.get_or_add_bool("mhd", "low_mach", False) is False


def test_config_defaults_and_ghosts():
    c = config_from_params(Params().read_text(TEXT))
    assert c["recon"] == 3 and c["rsolver"] == 1 and c["integrator"] == 3
    assert c["nghost"] == 3 and c["fofc"] == 0 and c["flatten"] == 1
    assert c["cfl"] == 0.3 and c["gamma"] == 5.0 / 3.0
    p = Params().read_text(TEXT)
    p.override("mhd.reconstruct=plm")
    assert config_from_params(p)["nghost"] == 2
    p.override("mesh.nghost=1")
    with pytest.raises(ParamError):
        config_from_params(p)


@pytest.mark.parametrize("key,val", [("mhd.reconstruct", "weno5"), ("mhd.rsolver", "roe"),
                                     ("time.integrator", "rk9"), ("mesh.bc_x1", "shear")])
def test_unknown_choices_raise(key, val):
    p = Params().read_text(TEXT)
    p.override(f"{key}={val}")
    with pytest.raises(ParamError):
        config_from_params(p)
