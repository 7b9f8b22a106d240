"""The differentiable mode's per-pair adjoint, on the CPU.

tests/native/diff_pair_check.cu instantiates the kernels' pair arithmetic
(autogrid_b200/csrc/kernels/diff_pair.cuh) in FP64 on the host and compares
the hand-written adjoint with central differences of the forward for random
atoms of every hbond class (D1 with each rexp, A1, ordered and disordered A2,
donor-acceptors), random bond vectors, the H-bond min/max terms and the
closest-hydrogen ramp.
"""
import shutil
import subprocess

import pytest

from conftest import ROOT

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = tmp_path_factory.mktemp("dpc") / "diff_pair_check"
    cmd = [NVCC, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", str(ROOT / "include"),
           "-I", str(ROOT / "autogrid_b200" / "csrc"), "-x", "cu",
           str(ROOT / "tests" / "native" / "diff_pair_check.cu"), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5, 6])
def test_pair_adjoint_matches_central_differences(checker, seed):
    r = subprocess.run([str(checker), str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
