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

Kink-free comparison (kink_free=True).  Almost every coordinate step of
1e-3 A moves some pair across a bin edge (the e map couples an atom to every
grid point), so no component is kink-free as a whole.  Instead, for each
checked component (atom a, axis i) and step h the check masks the grid points
at which L can have a kink along the stencil x -/+ h:
  * the pair (point, a) crosses a table bin edge, 128 r integer (this includes
    the 8 A cutoff and the EINTCLAMP plateau ends, which lie on bin edges), or
    for a disordered hydrogen a row-bin edge of 128 (r - 1.1);
  * the point lies within 8 A + 2h of an atom whose directional factors or
    H-bond min/max can switch as a moves: a itself, or an atom whose bond
    vectors depend on a, when any of them has an H-bond class.
On the remaining points L_m = sum m w maps is smooth along the stencil.  Its
adjoint is a backward with weights m w at the unmoved geometry; its central
difference comes from the same two forwards as the plain one.  Reported per h:
the norm-wise error over the components, the number of components with at
least one kink (all of them, typically) and the mean fraction of points
masked.
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


def _grid_points(problem: Problem) -> np.ndarray:
    n1, ne, sp = problem.n1, problem.ne, float(problem.scalars["spacing"])
    iz, iy, ix = np.meshgrid(np.arange(n1[2]), np.arange(n1[1]), np.arange(n1[0]), indexing="ij")
    return np.stack([(ix.ravel() - ne[0]) * sp, (iy.ravel() - ne[1]) * sp, (iz.ravel() - ne[2]) * sp], 1)


def _dependents(topo: np.ndarray) -> list:
    """deps[a]: atoms whose bond vectors depend on atom a's coordinates (a included)."""
    n = topo.shape[0]
    deps = [{a} for a in range(n)]
    for b in range(n):
        kind, i1, i2, nb = int(topo[b, 0]), int(topo[b, 1]), int(topo[b, 2]), int(topo[b, 3])
        if kind == 0:
            continue
        for j in [i1, i2] + [int(topo[b, 4 + k]) for k in range(max(0, min(nb, 3)))]:
            if 0 <= j < n:
                deps[j].add(b)
    return [sorted(d) for d in deps]


def kink_mask(problem: Problem, pts: np.ndarray, coord: np.ndarray, a: int, axis: int, h: float,
              deps: list) -> np.ndarray:
    """Points (bool [P]) at which L may have a slope kink as atom a moves by
    -/+ h along `axis` (see the module docstring)."""
    x0 = coord[a].copy()
    xm, xp = x0.copy(), x0.copy()
    xm[axis] -= h
    xp[axis] += h
    rm = np.linalg.norm(pts - xm, axis=1)
    rp = np.linalg.norm(pts - xp, axis=1)
    rlo, rhi = np.minimum(rm, rp), np.maximum(rm, rp)
    # the closest approach lies inside the stencil when the point's projection does
    inside = np.abs(pts[:, axis] - x0[axis]) < h
    perp = np.sqrt(np.maximum(rm * rm - (pts[:, axis] - xm[axis]) ** 2, 0.0))
    rlo = np.where(inside, np.minimum(rlo, perp), rlo)
    eps = 1e-9
    mask = (np.floor(128.0 * rlo - eps) != np.floor(128.0 * rhi + eps)) & (128.0 * rlo < 8191.0)
    dis = problem.arrays["disorder"]
    if int(problem.scalars.get("disorder_h", 0)) and dis is not None and dis[a] and \
            int(problem.arrays["rec_type"][a]) == int(problem.scalars.get("hydrogen_type", -1)):
        mask |= (np.floor(128.0 * (rlo - 1.10) - eps) != np.floor(128.0 * (rhi - 1.10) + eps)) & (rlo < 8.0 + h)
    hb = problem.arrays["hbond"]
    if any(int(hb[b]) != 0 for b in deps[a]):
        for b in deps[a]:
            mask |= np.linalg.norm(pts - coord[b], axis=1) < 8.0 + 2 * h
    return mask


def check(job: Job, problem: Problem, ctx: Context, atoms: np.ndarray, weights: np.ndarray,
          h_coord=(1e-3,), h_charge: float = 1e-4, kink_free: bool = False) -> dict:
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

        def maps_at(coord=None, charge=None):
            if coord is not None:
                rv, rv2 = job.bond_vectors(coord)
                d64.set_atoms(coord, charge0, rv, rv2)
            else:
                d64.set_atoms(coord0, charge, rv0, rv20)
            d64.forward(keep_closest_h=True)
            return d64.maps()

        def loss(coord=None, charge=None):
            return float(np.sum(w64 * maps_at(coord, charge)))

        t0 = time.perf_counter()
        hs = tuple(np.atleast_1d(h_coord).tolist())
        fd_c = {h: np.zeros((len(atoms), 3)) for h in hs}
        fd_q = np.zeros(len(atoms))
        if kink_free:
            pts = _grid_points(problem)
            deps = _dependents(job.bond_topology())
            masks = {}
            fdm_c = {h: np.zeros((len(atoms), 3)) for h in hs}
            kinked = {h: 0 for h in hs}
            masked_frac = {h: [] for h in hs}
        for k, a in enumerate(atoms):
            for h in hs:
                for i in range(3):
                    cp = coord0.copy(); cp[a, i] += h
                    cm = coord0.copy(); cm[a, i] -= h
                    mp = maps_at(coord=cp).copy()
                    mm = maps_at(coord=cm)
                    fd_c[h][k, i] = (float(np.sum(w64 * mp)) - float(np.sum(w64 * mm))) / (2 * h)
                    if kink_free:
                        bad = kink_mask(problem, pts, coord0, int(a), i, h, deps)
                        wm = w64 * (~bad).reshape((1,) + problem.map_shape[1:])
                        masks[(k, i, h)] = bad
                        fdm_c[h][k, i] = (float(np.sum(wm * mp)) - float(np.sum(wm * mm))) / (2 * h)
                        kinked[h] += int(bad.any())
                        masked_frac[h].append(float(bad.mean()))
            qp = charge0.copy(); qp[a] += h_charge
            qm = charge0.copy(); qm[a] -= h_charge
            fd_q[k] = (loss(charge=qp) - loss(charge=qm)) / (2 * h_charge)
        t_fd = time.perf_counter() - t0
        d64.set_atoms(coord0, charge0, rv0, rv20)
        if kink_free:
            # adjoint of each component's masked loss at the unmoved geometry
            d64.forward(keep_closest_h=True)
            gm_c = {h: np.zeros((len(atoms), 3)) for h in hs}
            for (k, i, h), bad in masks.items():
                wm = w64 * (~bad).reshape((1,) + problem.map_shape[1:])
                gc_m, _ = full_gradient(job, d64, coord0, wm)
                gm_c[h][k, i] = gc_m[atoms[k], i]
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
    if kink_free:
        out["fd_kink_free_coord"] = {h: _rel(gm_c[h], fdm_c[h]) for h in hs}
        out["fd_kinked_components"] = kinked
        out["fd_components"] = 3 * len(atoms)
        out["fd_masked_point_fraction"] = {h: float(np.mean(masked_frac[h])) for h in hs}
    return out
