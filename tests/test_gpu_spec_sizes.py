"""The batched, differentiable and Vina forms at the sizes of their workloads.

* batched ensemble: 256 seeded instances (atoms log-uniform 1,000-12,000,
  per-axis npts uniform 20-100, 8 maps), autotuned, graph-replayed: every
  instance within the parity bar of the FP64 oracle at 200 sampled points;
* differentiable maps: 4,000 atoms, 61^3 points, 8 maps, 64 random atoms:
  FP32 adjoint vs FP64 adjoint <= 1e-5; central differences at h = 1e-3 A on
  the kink-free part of the loss (autogrid_b200.gradcheck) <= 1e-3; charges
  (h = 1e-4 e) <= 1e-6;
* Vina conformers: 32 x 8,000 atoms, 101^3 points: the batched forward equals
  single-conformer forwards; the FP64 adjoint matches central differences at
  h = 1e-6 A.
"""
import os

import numpy as np
import pytest

from conftest import tolerance_ok

pytestmark = pytest.mark.gpu


def _load(d, gpf):
    from autogrid_b200 import Job
    cwd = os.getcwd()
    os.chdir(d)
    try:
        return Job(os.path.basename(str(gpf)), None)
    finally:
        os.chdir(cwd)


def test_batched_ensemble_256_instances(tmp_path, gpu_ctx):
    from autogrid_b200 import Batch, synth
    from oracle.oracle import oracle_points
    gpfs = synth.write_ensemble(tmp_path, 256, seed=2024)
    probs = [_load(tmp_path, g).problem() for g in gpfs]
    atoms = np.array([p.n_atoms for p in probs])
    assert atoms.min() >= 1000 and atoms.max() <= 12000
    assert {n for p in probs for n in p.n1} <= set(range(21, 102, 2))
    b = Batch(gpu_ctx, probs, autotune=True)
    b.run()
    b.run()  # graph replay
    rng = np.random.default_rng(5)
    for i, p in enumerate(probs):
        got = b.download(i).reshape(p.n_out, -1)
        pts = np.sort(rng.choice(p.points, 200, replace=False)).astype(np.int64)
        ref, flags = oracle_points(p, pts)
        ok = tolerance_ok(got[:p.n_maps, pts].astype(np.float64), ref) | (flags[None, :] != 0)
        assert ok.all(), f"instance {i}: {int((~ok).sum())} values outside the bar"
    t = b.tuning()
    assert t["candidates"] >= 4
    b.close()


def test_differentiable_4000_atoms_61cube(tmp_path, gpu_ctx):
    from autogrid_b200 import gradcheck, synth
    rec = synth.make_receptor(4000, seed=7, center=(0.0, 0.0, 0.0))
    g = synth.write_case(tmp_path, "c3", rec, synth.GridSpec(npts=(60, 60, 60)))
    job = _load(tmp_path, g)
    prob = job.problem()
    assert prob.n1 == (61, 61, 61) and prob.n_maps == 8
    rng = np.random.default_rng(3)
    w = rng.normal(size=prob.map_shape)
    atoms = rng.choice(prob.n_atoms, 64, replace=False)
    r = gradcheck.check(job, prob, gpu_ctx, atoms, w, h_coord=(1e-3,), kink_free=True)
    print({k: r[k] for k in ("fp32_vs_fp64_coord", "fp32_vs_fp64_charge", "fp64_vs_fd_charge",
                             "fp64_vs_fd_coord", "fd_kink_free_coord", "fd_kinked_components",
                             "fd_masked_point_fraction")})
    assert r["fp32_vs_fp64_coord"] <= 1e-5
    assert r["fp32_vs_fp64_charge"] <= 1e-5
    assert r["fp64_vs_fd_charge"] <= 1e-6
    assert r["fd_kink_free_coord"][1e-3] <= 1e-3
    assert r["fd_masked_point_fraction"][1e-3] < 0.5


def test_vina_32_conformers_8000_atoms_101cube(tmp_path, gpu_ctx):
    from autogrid_b200 import Diff, synth
    rec = synth.make_receptor(8000, seed=11, center=(0.0, 0.0, 0.0))
    types = ["A", "C", "F", "HD", "N", "NA", "OA", "SA"]
    g = synth.write_case(tmp_path, "c4", rec, synth.GridSpec(npts=(100, 100, 100), ligand_types=types))
    job = _load(tmp_path, g)
    vp = job.vina_problem()
    assert vp.n1 == (101, 101, 101) and vp.n_maps == 8
    rng = np.random.default_rng(4)
    base = vp.arrays["coord"].reshape(-1, 3)
    K = 32
    confs = [base + rng.normal(0.0, 0.3, base.shape) for _ in range(K)]
    df = Diff(gpu_ctx, vp, "fp32", conformers=K)
    for k, c in enumerate(confs):
        df.set_atoms(c, conformer=k)
    df.forward()
    batched = df.maps()
    for k in (0, 13, K - 1):
        one = Diff(gpu_ctx, vp, "fp32")
        one.set_atoms(confs[k])
        one.forward()
        assert np.array_equal(one.maps(), batched[k]), f"conformer {k}"
        one.close()
    df.close()
    # FP64 adjoint vs central differences at h = 1e-6 A on conformer 0
    d64 = Diff(gpu_ctx, vp, "fp64")
    d64.set_atoms(confs[0])
    d64.forward()
    w = rng.normal(size=vp.map_shape)
    gc = d64.backward(w)["coord"]  # Vina maps use no bond vectors
    h = 1e-6
    c0 = confs[0].copy()
    near = np.flatnonzero(np.all(np.abs(c0) < 18.0, axis=1))
    atoms = rng.choice(near, 4, replace=False)
    fd = np.zeros((len(atoms), 3))
    for k, a in enumerate(atoms):
        for i in range(3):
            cp = c0.copy(); cp[a, i] += h
            cm = c0.copy(); cm[a, i] -= h
            d64.set_atoms(cp); d64.forward(keep_closest_h=True); lp = float(np.sum(w * d64.maps()))
            d64.set_atoms(cm); d64.forward(keep_closest_h=True); lm = float(np.sum(w * d64.maps()))
            fd[k, i] = (lp - lm) / (2 * h)
    err = np.linalg.norm(gc[atoms] - fd) / np.linalg.norm(fd)
    assert err < 1e-3, err
    d64.close()
