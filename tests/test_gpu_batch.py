"""Batched ensemble (ag_batch_*): one persistent launch per kernel kind over
many uneven instances, autotuned and CUDA-graph captured; every instance's
maps must equal the single-instance path's within the parity tolerance and
match the FP64 oracle at sampled points."""
import os

import numpy as np
import pytest

from conftest import tolerance_ok

pytestmark = pytest.mark.gpu


def _load(tmp_path, gpfs):
    from autogrid_b200 import Job
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        return [Job(os.path.basename(g), None).problem() for g in gpfs]
    finally:
        os.chdir(cwd)


def test_batch_matches_single_and_oracle(tmp_path, gpu_ctx):
    from autogrid_b200 import Batch, synth
    from oracle.oracle import oracle_points
    gpfs = synth.write_ensemble(tmp_path, 7, seed=5, atoms_range=(150, 1500), npts_range=(4, 34), workers=1)
    probs = _load(tmp_path, gpfs)
    b = Batch(gpu_ctx, probs)
    tune = b.tuning()
    assert tune["candidates"] >= 9 and tune["far_tile"] in (256, 512, 1024) and tune["near_shape"] in (0, 1, 2)
    for rep in range(2):  # the captured graph replays
        b.run()
        rng = np.random.default_rng(rep)
        for i, p in enumerate(probs):
            got = b.download(i).reshape(p.n_maps, -1)
            single = gpu_ctx.compute(p).reshape(p.n_maps, -1)
            assert tolerance_ok(got, single).all(), f"instance {i}"
            pts = rng.choice(p.points, min(200, p.points), replace=False)
            ref, flags = oracle_points(p, pts)
            assert (tolerance_ok(got[:, pts], ref) | (flags[None, :] != 0)).all(), f"instance {i} vs oracle"
    b.close()


def test_batch_one_shot_and_errors(tmp_path, gpu_ctx):
    import ctypes as C
    from autogrid_b200 import AutoGridError, Batch, Problem, synth
    gpfs = synth.write_ensemble(tmp_path, 3, seed=9, atoms_range=(200, 400), npts_range=(4, 10), workers=1)
    probs = _load(tmp_path, gpfs)
    bad = Problem(**probs[1].arrays, n1=probs[1].n1, ne=(0, 0, 0), cov_pos=probs[1].cov_pos, **probs[1].scalars)
    with pytest.raises(AutoGridError) as e:
        Batch(gpu_ctx, [probs[0], bad, probs[2]])
    assert e.value.status == 1 and "instance 1" in e.value.message
    lib = gpu_ctx._lib
    from autogrid_b200._abi import ag_opts, ag_problem, check
    structs = [p.struct() for p in probs]
    arr = (C.POINTER(ag_problem) * 3)(*[C.pointer(s) for s in structs])
    outs = [np.empty(p.map_shape, dtype=np.float32) for p in probs]
    ptrs = (C.c_void_p * 3)(*[o.ctypes.data for o in outs])
    check(lib.ag_maps_compute_batch(gpu_ctx._h, arr, 3, C.byref(ag_opts()), ptrs))
    for p, o in zip(probs, outs):
        assert tolerance_ok(o, gpu_ctx.compute(p)).all()


def test_batch_one_shot_pipelined(tmp_path, gpu_ctx):
    """From 8 instances the one-shot call runs groups of instances as separate
    batches, building the next group while the previous one computes: the maps
    equal the single batch's bit for bit (same chunking, same summation order)
    and the per-box path's within the parity bar; errors name the caller's
    instance."""
    from autogrid_b200 import AutoGridError, Batch, Problem, synth
    from autogrid_b200.api import compute_batch
    gpfs = synth.write_ensemble(tmp_path, 10, seed=13, atoms_range=(150, 1200), npts_range=(4, 30), workers=1)
    probs = _load(tmp_path, gpfs)
    outs = compute_batch(gpu_ctx, probs)
    b = Batch(gpu_ctx, probs, autotune=False)
    b.run()
    for i, p in enumerate(probs):
        np.testing.assert_array_equal(outs[i], b.download(i))
        assert tolerance_ok(outs[i], gpu_ctx.compute(p)).all(), f"instance {i}"
    b.close()
    bad = Problem(**probs[6].arrays, n1=probs[6].n1, ne=(0, 0, 0), cov_pos=probs[6].cov_pos, **probs[6].scalars)
    with pytest.raises(AutoGridError) as e:
        compute_batch(gpu_ctx, probs[:6] + [bad] + probs[7:])
    assert e.value.status == 1 and "instance 6" in e.value.message
    # the groups' device blocks stay with the context until trimmed, and a
    # later call after the trim allocates afresh
    kept = gpu_ctx.cached_bytes()
    assert kept > 0
    assert gpu_ctx.trim() == kept and gpu_ctx.cached_bytes() == 0
    again = compute_batch(gpu_ctx, probs)
    for i in range(len(probs)):
        np.testing.assert_array_equal(again[i], outs[i])


def test_batch_with_distance_maps(tmp_path, gpu_ctx):
    """Instances asking for the floating and constriction grids get them after
    their energy maps, in the batch and in the one-shot batch call, equal to
    the single-instance path's (same FP64 kernel, computed once)."""
    from autogrid_b200 import Batch, synth
    from autogrid_b200.api import compute_batch
    from conftest import make_case
    probs = []
    for k, (n, npts) in enumerate([(300, (10, 12, 8)), (700, (16, 10, 14)), (500, (8, 8, 20))]):
        extra = ["fmap d%d.f.map" % k, "constriction_distance_cutoff 5.5", "cmap d%d.c.map" % k] if k != 1 else []
        probs.append(make_case(tmp_path, f"d{k}", n, npts, seed=40 + k, extra_lines=extra)[1])
    assert probs[0].n_out == probs[0].n_maps + 2 and probs[1].n_out == probs[1].n_maps
    singles = [gpu_ctx.compute(p) for p in probs]
    b = Batch(gpu_ctx, probs, autotune=False)
    b.run()
    for i, p in enumerate(probs):
        got = b.download(i)
        assert tolerance_ok(got[:p.n_maps], singles[i][:p.n_maps]).all()
        assert np.array_equal(got[p.n_maps:], singles[i][p.n_maps:])
    b.close()
    outs = compute_batch(gpu_ctx, probs * 3)  # 9 instances: the grouped one-shot path
    for i, o in enumerate(outs):
        p = probs[i % 3]
        assert np.array_equal(o[p.n_maps:], singles[i % 3][p.n_maps:])
