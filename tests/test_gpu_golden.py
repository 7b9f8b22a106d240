"""GPU maps against the reference's own full-precision output (tests/golden)
and the CLI drop-in against the reference's %.3f map files."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, tolerance_ok
from test_oracle_pinning import GOLDEN, full_precision_ok, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_fp32_matches_reference(path, tmp_path, gpu_ctx):
    from oracle.oracle import oracle_points
    z, job, prob = load_golden(path, tmp_path)
    ref = z["maps_full"]
    out = gpu_ctx.compute(prob, "fp32").reshape(prob.n_out, -1)
    got = out[:prob.n_maps]
    _, flags = oracle_points(prob)  # FP64-ambiguous points (bin edge within 1e-12) are exempt
    ok = tolerance_ok(got, ref) | (flags[None, :] != 0)
    bad = np.argwhere(~ok)
    assert bad.size == 0, f"{len(bad)} values outside 1e-3/1e-4; first {bad[:3].tolist()}"
    if "dist_full" in z.files:
        dist = out[prob.n_maps:]
        assert np.all(np.abs(dist[0] - z["dist_full"][0]) <= 1e-6 * np.abs(z["dist_full"][0]))
        assert np.array_equal(dist[1], z["dist_full"][1])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_fp64_twin_matches_reference(path, tmp_path, gpu_ctx):
    z, job, prob = load_golden(path, tmp_path)
    out = gpu_ctx.compute(prob, "fp64").reshape(prob.n_out, -1)
    assert full_precision_ok(out[:prob.n_maps], z["maps_full"]).all()
    if "dist_full" in z.files:
        dist = out[prob.n_maps:]
        assert np.all(np.abs(dist[0] - z["dist_full"][0]) <= 1.5e-7 * np.abs(z["dist_full"][0]))
        assert np.array_equal(dist[1], z["dist_full"][1])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_cli_drop_in(path, tmp_path, built):
    """autogrid4_b200 -p g.gpf -l g.glg writes the reference's .map and .fld files."""
    from oracle.oracle import read_map
    z = np.load(path, allow_pickle=False)
    (tmp_path / "g.gpf").write_text(str(z["gpf"]))
    (tmp_path / "g.pdbqt").write_text(str(z["pdbqt"]))
    cli = ROOT / "autogrid_b200" / "_build" / "autogrid4_b200"
    r = subprocess.run([str(cli), "-p", "g.gpf", "-l", "g.glg"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "Successful Completion" in "".join((tmp_path / "g.glg").read_text().splitlines()[-10:])
    for i, name in enumerate(z["names"]):
        mine = read_map(tmp_path / f"g.{name}.map")
        ref3 = z["maps_3dp"][i]
        full = z["maps_full"][i]
        # identical text except where our FP32 value rounds to the neighbouring 0.001 step,
        # or where a value within tolerance of the reference straddles the "0" threshold
        d = np.abs(mine - ref3)
        ok = (d <= 1.0005e-3) | tolerance_ok(mine, full)
        assert ok.all(), name
        # the reference prints (float)round3dp(e): a value's third decimal is only
        # stable against FP32 rounding (~6e-8 relative) well below 1e3, so the
        # byte-identical share is checked on |e| < 10 kcal/mol
        small = np.abs(full) < 10.0
        if small.sum() > 20:
            assert np.mean(d[small] == 0) > 0.9, name
    if "dist_names" in z.files:  # fmap text: %.3f of round3dp; cmap: integers
        for i, name in enumerate(z["dist_names"]):
            mine = read_map(tmp_path / f"g.{name}.map")
            assert np.all(np.abs(mine - z["dist_3dp"][i]) <= 1.0005e-3), name
        assert np.array_equal(read_map(tmp_path / "g.c.map"), z["dist_3dp"][1])
    drop = ("# Created by", "#GRID_PARAMETER_FILE")
    a = [ln for ln in (tmp_path / "g.maps.fld").read_text().splitlines() if not ln.startswith(drop)]
    b = [ln for ln in str(z["fld"]).splitlines() if not ln.startswith(drop)]
    assert a == b


def test_determinism_and_plan(tmp_path, gpu_ctx):
    from autogrid_b200 import Plan
    z, job, prob = load_golden(GOLDEN[0], tmp_path)
    a = gpu_ctx.compute(prob, "fp32")
    b = gpu_ctx.compute(prob, "fp32")
    assert np.array_equal(a, b)
    pl = Plan(gpu_ctx, prob)
    pl.run()
    pl.run()
    c = pl.download()
    pl.close()
    assert np.array_equal(a, c)


def test_status_codes(tmp_path, gpu_ctx):
    from autogrid_b200 import AutoGridError, Problem
    z, job, prob = load_golden(GOLDEN[0], tmp_path)
    # no DS/D1 hydrogen with ligand maps -> "no closestH atom was found" (main.cpp:3011-3014)
    kw = dict(prob.arrays)
    kw["hbond"] = np.where(np.isin(kw["hbond"], [1, 2]), 0, kw["hbond"]).astype(np.int32)
    bad = Problem(**kw, n1=prob.n1, ne=prob.ne, cov_pos=prob.cov_pos, **prob.scalars)
    with pytest.raises(AutoGridError) as e:
        gpu_ctx.compute(bad)
    assert e.value.status == 3
    # inconsistent grid
    bad2 = Problem(**prob.arrays, n1=prob.n1, ne=(0, 0, 0), cov_pos=prob.cov_pos, **prob.scalars)
    with pytest.raises(AutoGridError) as e:
        gpu_ctx.compute(bad2)
    assert e.value.status == 1
    # the context still works afterwards
    gpu_ctx.compute(prob)


def test_only_e_and_d_maps(tmp_path, gpu_ctx):
    """No ligand maps: the closest-H search is skipped, e and d still computed."""
    from autogrid_b200 import Problem
    from oracle.oracle import oracle_points
    z, job, prob = load_golden(GOLDEN[0], tmp_path)
    sc = dict(prob.scalars)
    sc.update(n_atom_maps=0, n_maps=2, elec_map=0, dsolv_map=1)
    p2 = Problem(**prob.arrays, n1=prob.n1, ne=prob.ne, cov_pos=prob.cov_pos, **sc)
    got = gpu_ctx.compute(p2).reshape(2, -1)
    ref, flags = oracle_points(p2)
    assert (tolerance_ok(got, ref) | (flags[None, :] != 0)).all()


COLLISION = sorted((ROOT / "tests" / "golden" / "collision").glob("*.npz"))


@pytest.mark.parametrize("path", COLLISION, ids=[p.stem for p in COLLISION])
def test_collision_mode_matches_bhtree_reference(path, tmp_path, gpu_ctx):
    """'map_receptor_interior off' on the GPU against the reference's USE_BHTREE
    build: e map (zero at the collision points), floating and constriction
    grids as the oracle pins them; every map within the parity bar; the FP64
    twin's e map to the printed float precision.  Batches and the
    differentiable mode refuse the mode."""
    from autogrid_b200 import AutoGridError, Batch, Diff
    z, job, prob = load_golden(path, tmp_path)
    names = [str(n) for n in z["names"]]
    for prec in ("fp32", "fp64"):
        out = gpu_ctx.compute(prob, prec).reshape(prob.n_out, -1)
        for k, n in enumerate(names):
            assert tolerance_ok(out[k].astype(np.float64), z["maps_full"][k]).all(), (prec, n)
        if "e" in names:
            e = names.index("e")
            assert np.array_equal(out[e] == 0, z["maps_full"][e] == 0), prec
            if prec == "fp64":
                assert full_precision_ok(out[e][None], z["maps_full"][e][None]).all()
        if z["dist_full"].size:
            nm = prob.n_maps
            assert np.all(np.abs(out[nm] - z["dist_full"][0]) <= 1e-6 * np.abs(z["dist_full"][0]) + 1e-6), prec
            assert np.array_equal(out[nm + 1], z["dist_full"][1]), prec
    for make in (lambda: Batch(gpu_ctx, [prob], autotune=False), lambda: Diff(gpu_ctx, prob, "fp32")):
        with pytest.raises(AutoGridError) as err:
            make()
        assert err.value.status == 4
