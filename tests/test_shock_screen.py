"""CPU check of the exact shock-threshold test of the detection kernels:
tests/native/shock_check.cpp compiles quotient_exceeds from the device header
with g++ and compares it with the plain IEEE division RN(a / m) > t on
random, near-threshold, screen-boundary and special values."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_screened_threshold_equals_the_division(tmp_path):
    exe = str(tmp_path / "shock_check")
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-std=c++17", "-I",
                           os.path.join(ROOT, "genasis_b200", "csrc"), "-o", exe,
                           os.path.join(ROOT, "tests", "native", "shock_check.cpp")], env=env)
    out = subprocess.check_output([exe], text=True).split("\n")
    cases, bad = map(int, [l for l in out if l and not l.startswith("#")][-1].split())
    assert cases > 1_000_000 and bad == 0, out[:12]
