"""Bond vectors at new coordinates (ag_job_bond_vectors) and their FP64
adjoint (ag_job_bond_vectors_backward), on the CPU.

* At the job's own coordinates the re-evaluation reproduces the problem's
  rvector/rvector2 bit for bit (main.cpp:2320-2656 arithmetic).
* The adjoint matches central differences of the re-evaluation for every
  bond-vector kind the receptors contain (D1 hydrogens, A1 nitrogens, A2
  acceptors with one or two bonded atoms, disordered hydroxyls).
"""
import os

import numpy as np
import pytest

from autogrid_b200 import Job, synth

CASES = [(1, False), (4, True), (6, True)]


def _job(tmp_path, seed, disorder_h):
    rec = synth.make_receptor(1500, seed=seed, radius=25.0)
    spec = synth.GridSpec(npts=(20, 20, 20), pre_lines=(["disorder_h"] if disorder_h else []))
    g = synth.write_case(tmp_path, "c", rec, spec)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        return Job(str(g), "c.glg")
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("seed,disorder_h", CASES)
def test_reevaluation_is_bit_identical(tmp_path, built, seed, disorder_h):
    job = _job(tmp_path, seed, disorder_h)
    p = job.problem()
    n = p.n_atoms
    rv, rv2 = job.bond_vectors()
    assert np.array_equal(rv, p.arrays["rvector"].reshape(n, 3))
    assert np.array_equal(rv2, p.arrays["rvector2"].reshape(n, 3))
    rv, rv2 = job.bond_vectors(p.arrays["coord"].reshape(n, 3).copy())
    assert np.array_equal(rv, p.arrays["rvector"].reshape(n, 3))
    assert np.array_equal(rv2, p.arrays["rvector2"].reshape(n, 3))
    # every directional class is present in these receptors
    hb = p.arrays["hbond"]
    assert (hb == 2).any() and (hb == 4).any() and (hb == 5).any()
    assert np.abs(rv2).sum() > 0


@pytest.mark.parametrize("seed,disorder_h", CASES)
def test_adjoint_matches_central_differences(tmp_path, built, seed, disorder_h):
    job = _job(tmp_path, seed, disorder_h)
    p = job.problem()
    n = p.n_atoms
    x0 = p.arrays["coord"].reshape(n, 3).copy()
    rng = np.random.default_rng(seed)
    g1 = rng.normal(size=(n, 3))
    g2 = rng.normal(size=(n, 3))

    def loss(x):
        rv, rv2 = job.bond_vectors(x)
        return float((g1 * rv).sum() + (g2 * rv2).sum())

    grad = job.bond_vectors_backward(x0, g1, g2)
    # atoms that move some bond vector, plus a few that do not
    moving = np.flatnonzero(np.abs(grad).sum(axis=1) > 0)
    assert moving.size > 50
    pick = np.concatenate([rng.choice(moving, 40, replace=False),
                           rng.choice(np.setdiff1d(np.arange(n), moving), 5, replace=False)])
    h = 1e-6
    fd = np.zeros((pick.size, 3))
    for k, a in enumerate(pick):
        for i in range(3):
            xp = x0.copy(); xp[a, i] += h
            xm = x0.copy(); xm[a, i] -= h
            fd[k, i] = (loss(xp) - loss(xm)) / (2 * h)
    an = grad[pick]
    err = np.abs(an - fd)
    assert np.all(err <= 1e-6 * np.maximum(1.0, np.abs(fd))), (err.max(), pick[np.argmax(err.max(axis=1))])
