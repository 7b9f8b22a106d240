"""The device map-text formatter, on the CPU.

tests/native/maptext_check.cpp compiles the formatter of
autogrid_b200/csrc/kernels/maptext.cuh as host code and compares every line
with the reference writer's own expression printed by glibc
(main.cpp:3481-3519: "0" below 1e-4, else "%.3f" of (float)round3dp(e) with
the 80-bit long double round3dp of main.cpp:84-86): halves of round(),
"%.3f" ties, quotients halfway between two floats, |e| >= 2^53, overflow to
inf, NaN, signed zero, counts, and seeded random values of every magnitude.
"""
import shutil
import subprocess

import pytest

from conftest import ROOT

CXX = shutil.which("g++")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if CXX is None:
        pytest.skip("g++ not found")
    out = tmp_path_factory.mktemp("mtc") / "maptext_check"
    cmd = [CXX, "-O2", "-std=c++17", "-I", str(ROOT / "include"), "-I", str(ROOT / "autogrid_b200" / "csrc"),
           str(ROOT / "tests" / "native" / "maptext_check.cpp"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_formatter_matches_glibc_reference_expression(checker, seed):
    r = subprocess.run([str(checker), str(seed), "200000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 mismatches" in r.stdout
