"""Vina-potential maps (ag_job_vina_problem) and conformer batches of the
differentiable mode, on the GPU.

* nearest-bin drop-in path on the Vina problem vs the FP64 oracle (plain sums,
  no e/d maps);
* linear-table FP64 twin vs the oracle's linear-mode restatement (1e-9), FP32
  within the drop-in bar;
* a batch of K jittered conformers in one launch equals K single evaluations
  (maps exactly, gradients to FP64 atomic-order rounding);
* the Vina adjoint against central differences, tightening as h shrinks.

Parity with the reference itself is unpinned: the reference compiles its Vina
path out (main.cpp:263).  The tables are pinned to main.cpp:2081-2126 as
written by tests/test_vina_tables.py.
"""
import numpy as np
import pytest

from conftest import make_case, tolerance_ok

pytestmark = pytest.mark.gpu

VINA_TYPES = ["A", "C", "F", "HD", "N", "NA", "OA", "SA"]


def _vina_case(tmp_path, n_atoms=500, npts=(14, 14, 14), seed=8):
    job, prob = make_case(tmp_path, "v", n_atoms, npts, seed=seed, radius=12.0, ligand_types=VINA_TYPES)
    return job, prob, job.vina_problem()


def test_vina_drop_in_matches_oracle(tmp_path, gpu_ctx):
    from oracle.oracle import oracle_points
    _, _, vp = _vina_case(tmp_path)
    assert vp.n_maps == len(VINA_TYPES)
    ref, flags = oracle_points(vp)
    got64 = gpu_ctx.compute(vp, "fp64").reshape(vp.n_maps, -1)
    ok = (np.abs(got64 - ref) <= 1e-9 * np.maximum(1, np.abs(ref))) | (flags[None, :] != 0)
    assert ok.all(), np.abs(got64 - ref).max()
    got32 = gpu_ctx.compute(vp, "fp32").reshape(vp.n_maps, -1)
    ok = tolerance_ok(got32, ref) | (flags[None, :] != 0)
    assert ok.all(), np.abs(got32 - ref).max()


def test_vina_linear_matches_oracle(tmp_path, gpu_ctx):
    from autogrid_b200 import Diff
    from oracle.oracle import oracle_points_lin
    _, _, vp = _vina_case(tmp_path)
    d64 = Diff(gpu_ctx, vp, "fp64")
    d64.forward()
    # no map reads Hramp: no closest-hydrogen search
    assert (d64.closest_h() == -1).all()
    ref = oracle_points_lin(vp, closest_h=np.full(vp.points, -1, np.int32))
    np.testing.assert_allclose(d64.maps().reshape(vp.n_maps, -1), ref, rtol=1e-9, atol=1e-9)
    d32 = Diff(gpu_ctx, vp, "fp32")
    d32.forward()
    ok = tolerance_ok(d32.maps().reshape(vp.n_maps, -1).astype(np.float64), ref)
    assert ok.all()
    d64.close(); d32.close()


@pytest.mark.parametrize("vina", [False, True])
def test_conformer_batch_equals_single_evaluations(tmp_path, gpu_ctx, vina):
    from autogrid_b200 import Diff
    job, prob, vp = _vina_case(tmp_path)
    p = vp if vina else prob
    K = 3
    rng = np.random.default_rng(5)
    base = p.arrays["coord"].reshape(-1, 3)
    confs = [base + rng.normal(0.0, 0.3, base.shape) for _ in range(K)]
    batch = Diff(gpu_ctx, p, "fp64", conformers=K)
    for k, c in enumerate(confs):
        rv, rv2 = job.bond_vectors(c)
        batch.set_atoms(c, None, rv, rv2, conformer=k)
    batch.forward()
    maps = batch.maps()
    w = rng.normal(size=batch.shape)
    gb = batch.backward(w)
    for k, c in enumerate(confs):
        single = Diff(gpu_ctx, p, "fp64")
        rv, rv2 = job.bond_vectors(c)
        single.set_atoms(c, None, rv, rv2)
        single.forward()
        np.testing.assert_array_equal(single.maps(), maps[k])
        gs = single.backward(w[k])
        for key in ("coord", "charge", "rvector", "rvector2"):
            np.testing.assert_allclose(gb[key][k], gs[key], rtol=1e-10, atol=1e-9)
        single.close()
    batch.close()


def test_vina_adjoint_matches_central_differences(tmp_path, gpu_ctx):
    from autogrid_b200 import gradcheck
    job, _, vp = _vina_case(tmp_path)
    rng = np.random.default_rng(12)
    w = rng.normal(size=vp.map_shape)
    c = vp.arrays["coord"].reshape(-1, 3)
    half = np.array(vp.ne) * vp.scalars["spacing"]
    near_box = np.flatnonzero(np.all(np.abs(c) < half + 4.0, axis=1))
    atoms = rng.choice(near_box, 16, replace=False)
    r = gradcheck.check(job, vp, gpu_ctx, atoms, w, h_coord=(1e-3, 1e-6))
    err = r["fp64_vs_fd_coord"]
    # The table as written steps by the H-bond weight at d = 0.7 and d = -0.7
    # and by the hydrophobic weight at d = 0.5; interpolated, each step is one
    # bin with a slope of ~75 kcal/mol/A, so a straddled bin edge costs a
    # finite difference ~100x more than in the AD4 tables.
    assert err[1e-6] < 1e-3, err
    assert err[1e-3] < 2e-1, err
    assert err[1e-6] < err[1e-3] / 20, err
    assert r["fp32_vs_fp64_coord"] < 1e-3, r["fp32_vs_fp64_coord"]
    # Vina maps do not depend on charges
    assert np.abs(r["fp64_charge"]).max() == 0.0
