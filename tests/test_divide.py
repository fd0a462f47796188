"""The division helpers of the flux kernel (chasqui_b200/csrc/chq_divide.cuh) return exactly
the IEEE quotient: built for the host with g++ (no contraction) and compared bit for bit on
special values, random doubles and floats over the whole exponent range, and every float
significand at both ends of the fast path (tests/div_check.cpp)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_div6_and_divz_equal_ieee_division(tmp_path):
    exe = tmp_path / "div_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", os.path.join(ROOT, "chasqui_b200", "csrc"),
                    "-o", str(exe), os.path.join(HERE, "div_check.cpp")], check=True)
    out = subprocess.run([str(exe), "5000000"], check=True, capture_output=True, text=True).stdout
    assert out.startswith("ok"), out
