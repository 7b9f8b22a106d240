"""Sharding a map set across ranks (autogrid_b200.shard), on the CPU.

z-slabs: two gloo ranks each compute their slab of a small problem with the
FP64 oracle; the stitched slabs equal the whole-grid oracle bit for bit.
Gradients: each rank computes its slab's partial dL/d(charge, coordinates) of
L = sum w * e (the differentiable e map: linearly interpolated
r_epsilon_fn over 1/max(r, 0.5)); one all-reduce gives the whole grid's
gradient.  Instances: the greedy split covers every instance once and
balances the cost.
"""
import json
import os
import socket
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT, make_case


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(tmp_path, body: str, world: int = 2, timeout: int = 240) -> list:
    """Run `body` (defines main(rank, world) -> json-able) on `world` gloo
    ranks on 127.0.0.1; returns the results by rank."""
    script = tmp_path / "ranks.py"
    script.write_text(textwrap.dedent("""
        import os, sys, json
        sys.path.insert(0, {root!r})
        sys.path.insert(0, {tests!r})
        import torch.distributed as dist
    """).format(root=str(ROOT), tests=str(ROOT / "tests")) + textwrap.dedent(body) + textwrap.dedent("""
        if __name__ == "__main__":
            rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
            dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
            res = main(rank, world)
            dist.barrier()
            dist.destroy_process_group()
            print("RESULT " + json.dumps(res))
    """))
    port = str(_free_port())
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=port, CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, cwd=str(tmp_path),
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        o, e = p.communicate(timeout=timeout)
        assert p.returncode == 0, e[-3000:]
        line = [ln for ln in o.splitlines() if ln.startswith("RESULT ")][-1]
        out.append(json.loads(line[7:]))
    return out


def test_zslab_ranges_cover_the_grid_aligned():
    from autogrid_b200.shard import zslab_ranges
    for n1z in (1, 7, 8, 9, 41, 127, 128, 201):
        for world in (1, 2, 3, 4, 8):
            r = zslab_ranges(n1z, world)
            assert len(r) == world
            assert r[0][0] == 0 and r[-1][1] == n1z
            for (a0, a1), (b0, b1) in zip(r, r[1:]):
                assert a1 == b0
            for z0, z1 in r:
                assert z0 <= z1 and z0 % 8 == 0 and (z1 % 8 == 0 or z1 == n1z)
    # 127 planes on 8 ranks: two frame rows each, the last one 15 planes
    assert zslab_ranges(127, 8) == [(0, 16), (16, 32), (32, 48), (48, 64), (64, 80), (80, 96), (96, 112),
                                    (112, 127)]


def test_partition_instances_balanced_and_complete():
    from autogrid_b200.shard import partition_instances
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0, 1.5, 256)
    for world in (1, 2, 4, 8):
        parts = partition_instances(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: no rank exceeds the mean by more than the largest instance
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
        assert parts == partition_instances(costs, world)  # deterministic


def test_zslab_problem_keeps_point_coordinates(tmp_path, built):
    """The oracle at a slab sub-problem's points equals the oracle at the
    same points of the whole grid (the same coordinates, bit for bit)."""
    from autogrid_b200.shard import zslab_problem
    from oracle.oracle import oracle_points
    _, prob = make_case(tmp_path, "slab", 150, (6, 8, 10), seed=2, radius=7.0)
    whole, _ = oracle_points(prob)
    whole = whole.reshape(prob.n_maps, prob.n1[2], -1)
    for z0, z1 in ((0, 3), (3, 11), (5, 6)):
        sub, _ = oracle_points(zslab_problem(prob, z0, z1))
        assert np.array_equal(sub.reshape(prob.n_maps, z1 - z0, -1), whole[:, z0:z1])


SLAB_BODY = """
    import numpy as np
    from pathlib import Path
    from conftest import make_case
    from autogrid_b200.shard import zslab_ranges, zslab_problem, stitch_zslabs
    from oracle.oracle import oracle_points

    def main(rank, world):
        d = Path(f"r{rank}"); d.mkdir(exist_ok=True)
        _, prob = make_case(d, "w", 220, (8, 10, 20), seed=11, radius=8.0)
        ranges = zslab_ranges(prob.n1[2], world)
        z0, z1 = ranges[rank]
        mine, _ = oracle_points(zslab_problem(prob, z0, z1))
        parts = [None] * world
        dist.all_gather_object(parts, mine.tolist())
        if rank != 0:
            return {"rank": rank}
        slabs = [np.asarray(p).reshape(prob.n_maps, r[1] - r[0], prob.n1[1], prob.n1[0])
                 for p, r in zip(parts, ranges)]
        got = stitch_zslabs(slabs, ranges, prob.n_maps, prob.n1)
        whole, _ = oracle_points(prob)
        return {"rank": 0, "equal": bool(np.array_equal(got.reshape(prob.n_maps, -1), whole)),
                "ranges": ranges}
"""


def test_two_gloo_ranks_compute_zslabs_that_stitch_to_the_whole(tmp_path, built):
    res = run_ranks(tmp_path, SLAB_BODY)
    r0 = next(r for r in res if r["rank"] == 0)
    assert r0["ranges"] == [[0, 8], [8, 21]]
    assert r0["equal"]


GRAD_BODY = """
    import numpy as np
    import torch
    from pathlib import Path
    from conftest import make_case
    from autogrid_b200.shard import zslab_ranges, zslab_problem, allreduce_gradients

    def emap_grad(prob, w):
        # dL/dq and dL/dx of L = sum_p w_p e_p, e_p = sum_a q_a coeff T(128 r)/max(r, 0.5),
        # T linearly interpolated in r_epsilon_fn (the differentiable mode's e map)
        xyz = prob.arrays["coord"].reshape(-1, 3)
        q = prob.arrays["charge"]
        T = prob.arrays["r_epsilon_fn"]
        coeff = float(prob.scalars["coeff_estat"])
        sp = float(prob.scalars["spacing"])
        n1, ne = prob.n1, prob.ne
        iz, iy, ix = np.meshgrid(*[np.arange(n) for n in n1[::-1]], indexing="ij")
        c = np.stack([(ix.ravel() - ne[0]) * sp, (iy.ravel() - ne[1]) * sp, (iz.ravel() - ne[2]) * sp], 1)
        d = xyz[None, :, :] - c[:, None, :]
        r = np.sqrt((d * d).sum(-1))
        x = np.minimum(r * 128.0, 8191.0)
        b = np.minimum(np.floor(x).astype(int), 8190)
        f = x - b
        Tx = T[b] + f * (T[b + 1] - T[b])
        dT = np.where(r * 128.0 < 8191.0, (T[b + 1] - T[b]) * 128.0, 0.0)
        rm = np.maximum(r, 0.5)
        g = Tx / rm
        dg = dT / rm - np.where(r > 0.5, Tx / (rm * rm), 0.0)
        wv = w.reshape(-1)[:, None]
        gq = coeff * (wv * g).sum(0)
        gx = coeff * q[None, :, None] * (wv * dg)[:, :, None] * d / np.maximum(r, 1e-12)[:, :, None]
        return gq, gx.sum(0)

    def main(rank, world):
        d = Path(f"g{rank}"); d.mkdir(exist_ok=True)
        _, prob = make_case(d, "g", 60, (6, 6, 17), seed=4, radius=6.0)
        w = np.random.default_rng(9).standard_normal(prob.points).reshape(prob.n1[2], -1)
        z0, z1 = zslab_ranges(prob.n1[2], world)[rank]
        gq, gx = emap_grad(zslab_problem(prob, z0, z1), w[z0:z1])
        tq, tx = torch.from_numpy(gq.copy()), torch.from_numpy(gx.copy())
        allreduce_gradients([tq, tx])
        fq, fx = emap_grad(prob, w)
        scale = max(np.abs(fq).max(), np.abs(fx).max())
        err = max(np.abs(tq.numpy() - fq).max(), np.abs(tx.numpy() - fx).max()) / scale
        part = max(np.abs(gq - fq).max(), np.abs(gx - fx).max()) / scale
        return {"rank": rank, "err": float(err), "partial_differs": float(part)}
"""


def test_two_gloo_ranks_allreduce_slab_gradients(tmp_path, built):
    res = run_ranks(tmp_path, GRAD_BODY)
    for r in res:
        assert r["err"] < 1e-12, r
        assert r["partial_differs"] > 1e-6, r  # each rank alone holds only part of the gradient
