"""GPU parity against the FP64 oracle (a C restatement of main.cpp:2805-3464).

Bar: |gpu - oracle| <= max(1e-3, 1e-4*|oracle|) kcal/mol for the FP32 path, at
every point except those the oracle flags as FP64-ambiguous (a pair within
1e-12 of a bin edge / cutoff / branch); the FP64 twin must agree to 1e-9.
"""
import numpy as np
import pytest

from conftest import make_case, tolerance_ok

pytestmark = pytest.mark.gpu


def _check(prob, maps_gpu, points=None, rel=1e-4, abs_=1e-3):
    from oracle.oracle import oracle_points
    ref, flags = oracle_points(prob, points)
    got = maps_gpu.reshape(prob.n_maps, -1)
    if points is not None:
        got = got[:, points]
    ok = tolerance_ok(got, ref, abs_, rel) | (flags[None, :] != 0)
    bad = np.argwhere(~ok)
    assert bad.size == 0, f"{len(bad)} mismatches; first {bad[:5].tolist()} got {got[tuple(bad[0])]} ref {ref[tuple(bad[0])]}"
    return ref, flags


@pytest.mark.parametrize("seed", [1, 2])
def test_small_box_fp32_all_points(tmp_path, gpu_ctx, seed):
    _, prob = make_case(tmp_path, "s", 400, (10, 12, 14), seed=seed, radius=11.0)
    maps = gpu_ctx.compute(prob, "fp32")
    _check(prob, maps)
    st = gpu_ctx.stats()
    assert st.near_pairs > 0 and st.gpu_launches >= 2


@pytest.mark.parametrize("seed", [1, 2])
def test_small_box_fp64_twin_all_points(tmp_path, gpu_ctx, seed):
    _, prob = make_case(tmp_path, "s", 400, (10, 12, 14), seed=seed, radius=11.0)
    maps = gpu_ctx.compute(prob, "fp64")
    _check(prob, maps, rel=1e-9, abs_=1e-9)


def test_config0_sampled_points(tmp_path, gpu_ctx):
    _, prob = make_case(tmp_path, "c0", 1800, (40, 40, 40), seed=0, radius=28.0)
    maps = gpu_ctx.compute(prob, "fp32")
    rng = np.random.default_rng(0)
    pts = rng.choice(prob.points, 3000, replace=False)
    _check(prob, maps, pts)
