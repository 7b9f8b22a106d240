"""Splitting map work across GPUs: one process per GPU, torch.distributed.

The map loop has no exchange step.  Every grid point needs every atom but no
other point, so a map set splits by z-slab of the grid (the axis the
reference's OpenMP loop splits, main.cpp:2805) and a batch of independent
receptor/box instances splits by instance.  Neither needs a collective on the
data path.  The differentiable mode's adjoint is the one exception: each
rank's slab contributes a partial dL/d(coordinates, charges) over all atoms,
and the ranks sum them with one all-reduce (allreduce_gradients).

Functions here are host logic only (no kernels); they are covered by
world-size-2 gloo tests on the CPU.
"""
from __future__ import annotations

import numpy as np

from .api import Problem

FRAME_Z = 8  # z-slab bounds of ag_maps_compute_zslab: multiples of 8 planes (or the last plane)


def zslab_ranges(n1z: int, world: int, align: int = FRAME_Z) -> list[tuple[int, int]]:
    """Split planes [0, n1z) into `world` contiguous slabs whose bounds are
    multiples of `align` (the last ends at n1z), as even in planes as the
    alignment allows.  A rank may get an empty slab (z0 == z1) when there are
    fewer aligned blocks than ranks."""
    if world < 1 or n1z < 0:
        raise ValueError("world >= 1 and n1z >= 0")
    blocks = (n1z + align - 1) // align
    out = []
    for r in range(world):
        b0 = (blocks * r) // world
        b1 = (blocks * (r + 1)) // world
        out.append((min(b0 * align, n1z), min(b1 * align, n1z)))
    return out


def zslab_problem(problem: Problem, z0: int, z1: int) -> Problem:
    """The sub-problem of planes [z0, z1): the same atoms and tables on a grid
    of z1 - z0 planes whose first plane is plane z0.  Grid coordinates are
    (i - ne) * spacing (main.cpp:2859); with i' = i - z0 and ne' = ne - z0
    every point keeps its coordinate exactly, so the slab's maps are the
    whole grid's maps at those planes."""
    if not (0 <= z0 < z1 <= problem.n1[2]):
        raise ValueError("slab outside the grid or empty")
    kw = dict(problem.arrays)
    kw.update(problem.scalars)
    kw["n1"] = (problem.n1[0], problem.n1[1], z1 - z0)
    kw["ne"] = (problem.ne[0], problem.ne[1], problem.ne[2] - z0)
    kw["cov_pos"] = problem.cov_pos
    return Problem(**kw)


def instance_cost(problem: Problem) -> float:
    """Relative cost of one instance: points x (atoms + 64), the measure the
    batch orders its work by (far-field pairs plus per-point near work)."""
    return float(problem.points) * (problem.n_atoms + 64)


def partition_instances(costs, world: int) -> list[list[int]]:
    """Deterministic greedy longest-processing-time split of instances over
    ranks: instances by decreasing cost (ties by index), each to the rank with
    the least total so far (ties to the lowest rank).  Returns each rank's
    instance indices in increasing order."""
    costs = [float(c) for c in costs]
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def stitch_zslabs(slabs, ranges, n_out: int, n1: tuple) -> np.ndarray:
    """Whole-grid maps [n_out, n1z, n1y, n1x] from per-slab maps
    [n_out, z1 - z0, n1y, n1x] and their ranges."""
    out = np.empty((n_out, n1[2], n1[1], n1[0]), dtype=np.asarray(slabs[0]).dtype)
    for s, (z0, z1) in zip(slabs, ranges):
        if z1 > z0:
            out[:, z0:z1] = s
    return out


def allreduce_gradients(grads, group=None):
    """Sum per-rank gradient partials over all ranks with one all-reduce:
    the tensors are packed into one flat buffer (same dtype and device),
    reduced in place, and unpacked back into the given tensors.  Returns them."""
    import torch
    import torch.distributed as dist
    grads = list(grads)
    if not grads:
        return grads
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return grads
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for g in grads:
        n = g.numel()
        g.copy_(flat[off:off + n].view_as(g))
        off += n
    return grads
