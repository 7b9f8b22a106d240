"""Sharded map sets on the GPU: z-slabs and partial gradients.

* ag_maps_compute_zslab: the slabs of a map set equal the one-shot call's
  planes bit for bit (every map, the e map included);
* ag_plan_run_zslab: a plan run slab by slab leaves the same device maps as
  ag_plan_run;
* the differentiable mode on z-slab sub-problems (what each rank of a
  sharded adjoint computes): the per-slab gradients sum to the whole grid's.
"""
import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(tmp_path_factory, built):
    d = tmp_path_factory.mktemp("shard")
    return make_case(d, "s", 1500, (36, 30, 40), seed=21, radius=16.0)


def test_zslabs_equal_one_shot_bit_for_bit(case, gpu_ctx):
    from autogrid_b200.shard import stitch_zslabs, zslab_ranges
    _, prob = case
    whole = gpu_ctx.compute(prob, "fp32")
    for world in (2, 3, 5):
        ranges = zslab_ranges(prob.n1[2], world)
        slabs = [gpu_ctx.compute_zslab(prob, z0, z1) for z0, z1 in ranges]
        got = stitch_zslabs(slabs, ranges, prob.n_out, prob.n1)
        assert np.array_equal(got, whole), f"world {world}"


def test_zslab_bounds_are_checked(case, gpu_ctx):
    from autogrid_b200 import AutoGridError
    _, prob = case
    for z0, z1 in ((4, 16), (0, 12), (8, 8), (0, prob.n1[2] + 1)):
        with pytest.raises(AutoGridError):
            gpu_ctx.compute_zslab(prob, z0, z1)


def test_plan_zslab_runs_equal_plan_run(case, gpu_ctx):
    from autogrid_b200.shard import zslab_ranges
    _, prob = case
    plan = gpu_ctx.plan(prob)
    plan.run()
    ref = plan.download().copy()
    plan2 = gpu_ctx.plan(prob)
    for z0, z1 in zslab_ranges(prob.n1[2], 3):
        plan2.run_zslab(z0, z1)
    got = plan2.download()
    assert np.array_equal(got, ref)
    plan.close()
    plan2.close()


def test_sharded_adjoint_gradients_sum_to_whole(tmp_path, gpu_ctx):
    """FP64 twin: gradients of L = sum w * maps over each slab, summed over the
    slabs, equal the whole grid's (summation order only)."""
    import torch
    from autogrid_b200.shard import zslab_ranges
    from autogrid_b200.torch_maps import GridMaps
    job, prob = make_case(tmp_path, "g", 500, (14, 12, 22), seed=8, radius=11.0)
    rng = np.random.default_rng(2)
    w = torch.from_numpy(rng.standard_normal(prob.map_shape)).cuda()
    c0 = torch.from_numpy(prob.arrays["coord"].reshape(-1, 3).copy())
    q0 = torch.from_numpy(prob.arrays["charge"].copy())

    def grads(zslab):
        f = GridMaps(job, 0, "fp64", zslab=zslab)
        c = c0.clone().cuda().requires_grad_(True)
        q = q0.clone().cuda().requires_grad_(True)
        m = f(c, q)
        ww = w if zslab is None else w[:, zslab[0]:zslab[1]]
        (ww * m).sum().backward()
        return c.grad.cpu().numpy(), q.grad.cpu().numpy()

    gc, gq = grads(None)
    sc, sq = np.zeros_like(gc), np.zeros_like(gq)
    for z0, z1 in zslab_ranges(prob.n1[2], 3):
        a, b = grads((z0, z1))
        sc += a
        sq += b
    assert np.abs(sc - gc).max() <= 1e-10 * np.abs(gc).max()
    assert np.abs(sq - gq).max() <= 1e-10 * np.abs(gq).max()


def test_collision_mode_zslabs_equal_one_shot(tmp_path, gpu_ctx):
    """'map_receptor_interior off' on z-slabs: the collision rule runs on each
    slab's planes, so the slabs (energy maps, floating and constriction grids)
    equal the one-shot call's planes bit for bit."""
    from autogrid_b200.shard import stitch_zslabs, zslab_ranges
    _, prob = make_case(tmp_path, "coll", 900, (14, 12, 26), seed=23, radius=11.0,
                        ligand_types=["A", "C", "HD", "OA"],
                        extra_lines=["map_receptor_interior off", "fmap c.f.map", "constriction_distance_cutoff 5.5",
                                     "cmap c.c.map"])
    assert int(prob.scalars.get("report_collisions", 0)) == 1 and prob.n_out == prob.n_maps + 2
    whole = gpu_ctx.compute(prob, "fp32")
    e = int(prob.scalars["elec_map"])
    assert (whole[e] == 0).any()  # some points collide
    ranges = zslab_ranges(prob.n1[2], 2)
    slabs = [gpu_ctx.compute_zslab(prob, z0, z1) for z0, z1 in ranges]
    got = stitch_zslabs(slabs, ranges, prob.n_out, prob.n1)
    assert np.array_equal(got, whole)
