"""Check the differentiable mode's adjoint against central differences.

For L = sum(w * maps) with fixed weights w, compares on chosen atoms
  * the FP64 adjoint (ag_diff_backward on the FP64 twin, plus the FP64
    bond-vector chain ag_job_bond_vectors_backward) with central differences
    of L evaluated by the FP64 twin forward (h on a coordinate or a charge; the
    bond vectors recomputed at every displaced geometry with the frozen
    neighbours; each point's closest DS/D1 atom frozen);
  * the FP32 adjoint with the FP64 adjoint.
Errors are norm-wise relative over the checked components:
||a - b||_2 / ||b||_2.

The mode's tables are piecewise linear in A_DIV r (bins of 1/128 A), so L has
a slope kink wherever a pair distance crosses a bin edge.  A central
difference with h comparable to the bin width averages the slopes on both
sides of every kink the step crosses, which the point derivative does not: the
difference between the adjoint and such a finite difference shrinks in
proportion to h.  `h_coord` may therefore list several steps; each gets its
own comparison.
"""
from __future__ import annotations

import time

import numpy as np

from .api import Context, Diff, Job, Problem


def full_gradient(job: Job, diff: Diff, coord: np.ndarray, weights: np.ndarray) -> tuple:
    """(dL/dcoord [N,3], dL/dcharge [N]) of the last forward of `diff`."""
    g = diff.backward(weights.astype(diff.dtype, copy=False))
    gc = g["coord"] + job.bond_vectors_backward(coord, g["rvector"], g["rvector2"])
    return gc, g["charge"]


def _rel(a: np.ndarray, b: np.ndarray) -> float:
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / nb if nb > 0 else float(np.linalg.norm(a))


def check(job: Job, problem: Problem, ctx: Context, atoms: np.ndarray, weights: np.ndarray,
          h_coord=(1e-3,), h_charge: float = 1e-4) -> dict:
    n = problem.n_atoms
    coord0 = problem.arrays["coord"].reshape(n, 3).copy()
    charge0 = problem.arrays["charge"].copy()
    w64 = np.ascontiguousarray(weights, dtype=np.float64).reshape(problem.map_shape)
    d64 = Diff(ctx, problem, "fp64")
    d32 = Diff(ctx, problem, "fp32")
    try:
        d64.forward()
        d32.forward()
        t_fwd32, t_ch32, _ = d32.timing()
        g64c, g64q = full_gradient(job, d64, coord0, w64)
        g32c, g32q = full_gradient(job, d32, coord0, w64)
        _, _, t_bwd32 = d32.timing()
        rv0, rv20 = job.bond_vectors(coord0)

        def loss(coord=None, charge=None):
            if coord is not None:
                rv, rv2 = job.bond_vectors(coord)
                d64.set_atoms(coord, charge0, rv, rv2)
            else:
                d64.set_atoms(coord0, charge, rv0, rv20)
            d64.forward(keep_closest_h=True)
            return float(np.sum(w64 * d64.maps()))

        t0 = time.perf_counter()
        hs = tuple(np.atleast_1d(h_coord).tolist())
        fd_c = {h: np.zeros((len(atoms), 3)) for h in hs}
        fd_q = np.zeros(len(atoms))
        for k, a in enumerate(atoms):
            for h in hs:
                for i in range(3):
                    cp = coord0.copy(); cp[a, i] += h
                    cm = coord0.copy(); cm[a, i] -= h
                    fd_c[h][k, i] = (loss(coord=cp) - loss(coord=cm)) / (2 * h)
            qp = charge0.copy(); qp[a] += h_charge
            qm = charge0.copy(); qm[a] -= h_charge
            fd_q[k] = (loss(charge=qp) - loss(charge=qm)) / (2 * h_charge)
        t_fd = time.perf_counter() - t0
        d64.set_atoms(coord0, charge0, rv0, rv20)
    finally:
        d64.close()
        d32.close()
    a = np.asarray(atoms)
    out = {
        "atoms": a, "h_coord": hs, "h_charge": h_charge,
        "fd_coord": fd_c, "fd_charge": fd_q,
        "fp64_coord": g64c[a], "fp64_charge": g64q[a],
        "fp32_coord": g32c[a], "fp32_charge": g32q[a],
        "fp64_vs_fd_coord": {h: _rel(g64c[a], fd_c[h]) for h in hs},
        "fp32_vs_fd_coord": {h: _rel(g32c[a], fd_c[h]) for h in hs},
        "fp64_vs_fd_charge": _rel(g64q[a], fd_q), "fp32_vs_fd_charge": _rel(g32q[a], fd_q),
        "fp32_vs_fp64_coord": _rel(g32c, g64c), "fp32_vs_fp64_charge": _rel(g32q, g64q),
        "fp32_forward_ms": t_fwd32, "fp32_closest_h_ms": t_ch32, "fp32_backward_ms": t_bwd32,
        "fd_seconds": t_fd, "fd_evaluations": 2 * len(atoms) * (3 * len(hs) + 1),
    }
    return out
