"""Map-file text formatted on the device (ag_maps_format, ag_maps_compute_text,
ag_job_write_text) against the host writer, which prints with glibc exactly as
the reference does (main.cpp:3481-3519).

* every golden case, FP32 and FP64: the map files written from device text are
  byte-identical to the host writer's files for the same maps, and the GLG
  extrema tables agree;
* edge values written into device maps (halves of round3dp, "%.3f" ties,
  values straddling the 1e-4 zero rule, huge values, inf/NaN, counts) format
  as glibc formats the reference's expression;
* a plan's device maps format to the same text as the one-shot call;
* the CLI with the device writer and with --host-writer write the same files.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_oracle_pinning import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def _map_files(d):
    return sorted(p for p in d.iterdir() if p.suffix == ".map")


def _extrema_table(glg):
    lines = glg.read_text().splitlines()
    i = next(k for k, l in enumerate(lines) if l.startswith("Grid\tAtom"))
    j = next(k for k, l in enumerate(lines) if "Every pairwise-atomic interaction" in l)
    return lines[i:j]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_device_text_matches_host_writer(path, tmp_path, gpu_ctx, precision):
    da, db = tmp_path / "dev", tmp_path / "host"
    da.mkdir(); db.mkdir()
    _, job_a, prob = load_golden(path, da)
    _, job_b, _ = load_golden(path, db)
    mt = gpu_ctx.compute_text(prob, precision)
    assert mt.map_bytes.shape == (prob.n_out,)
    maps = gpu_ctx.compute(prob, precision)
    job_a.write_text(mt)
    job_b.write_maps(maps)
    job_a.close(); job_b.close()
    fa, fb = _map_files(da), _map_files(db)
    assert [p.name for p in fa] == [p.name for p in fb] and fa
    for a, b in zip(fa, fb):
        ta, tb = a.read_bytes(), b.read_bytes()
        assert ta == tb, f"{a.name}: first difference at byte {next(i for i in range(min(len(ta), len(tb))) if ta[i] != tb[i]) if len(ta) == len(tb) else 'length'}"
    assert _extrema_table(da / "g.glg") == _extrema_table(db / "g.glg")
    flat = maps.reshape(prob.n_out, -1).astype(np.float64)
    np.testing.assert_array_equal(mt.emin, flat[:prob.n_maps].min(axis=1))
    np.testing.assert_array_equal(mt.emax, flat[:prob.n_maps].max(axis=1))


def _ref_line(kind, e):
    """The reference's writer expression, main.cpp:3481-3519 with round3dp of
    main.cpp:84-86 in 80-bit long double."""
    if kind == 2:
        return "%d\n" % int(e)
    if kind == 0 and abs(e) < 0.0001:
        return "0\n"
    if np.isnan(e):
        return ("-nan\n" if np.signbit(e) else "nan\n")
    if np.isinf(e):
        return ("-inf\n" if e < 0 else "inf\n")
    x = np.longdouble(e) * np.longdouble(1000)
    r = np.copysign(np.floor(np.abs(x) + np.longdouble(0.5)), x) if abs(e) < 2.0 ** 52 else x
    v = np.float32(r / np.longdouble(1000))
    if np.isinf(v):
        return ("-inf\n" if v < 0 else "inf\n")
    return "%.3f\n" % float(v)


def _edge_values(rng, n):
    fixed = [0.0, -0.0, 1e-4, -1e-4, np.nextafter(1e-4, 0), np.nextafter(-1e-4, 0), 0.0005, -0.0005, 0.0625,
             -0.0625, 16384.0625, -16384.0625, 1e12, -1e12, 1e15, 9.5e15, 1e20, -3.3e38, 3.5e38, np.inf, -np.inf,
             np.nan, 123.4565, 0.9995, 1.0005, -1.0005, 5e-324, 99999.9995]
    halves = (rng.integers(-2**29, 2**29, n) / 2.0 ** rng.integers(1, 15, n))
    ticks = (rng.integers(-10**8, 10**8, n) + 0.5) / 1000.0
    logu = np.sign(rng.standard_normal(n)) * 10.0 ** rng.uniform(-7, 16, n)
    return np.concatenate([np.array(fixed), halves, ticks, logu, 200 * (rng.random(n) - 0.5)])


@pytest.mark.parametrize("elem", [4, 8])
def test_device_text_edge_values(tmp_path, gpu_ctx, elem):
    import torch
    path = next(p for p in GOLDEN if p.stem == "distance_maps")
    _, job, prob = load_golden(path, tmp_path)
    job.close()
    P = prob.points
    assert prob.n_out == prob.n_maps + 2  # floating and constriction maps
    rng = np.random.default_rng(5)
    vals = _edge_values(rng, 4 * P)
    maps = np.empty((prob.n_out, P))
    for k in range(prob.n_maps):
        maps[k] = np.resize(np.roll(vals, 977 * k), P)
    maps[prob.n_maps] = np.resize(np.abs(vals), P)
    maps[prob.n_maps + 1] = rng.integers(0, 5000, P)
    if elem == 4:
        with np.errstate(over="ignore"):
            maps = maps.astype(np.float32)
    dev = torch.from_numpy(np.ascontiguousarray(maps)).cuda()
    torch.cuda.synchronize()
    mt = gpu_ctx.format(prob, dev.data_ptr(), elem)
    kinds = [0] * prob.n_maps + [1, 2]
    bad = []
    for k in range(prob.n_out):
        got = mt.body(k).decode().splitlines(keepends=True)
        ref = [_ref_line(kinds[k], float(e)) for e in maps[k]]
        assert len(got) == len(ref)
        bad += [(k, float(maps[k][i]), got[i], ref[i]) for i in range(len(ref)) if got[i] != ref[i]]
    assert not bad, bad[:10]
    flat = maps[:prob.n_maps].astype(np.float64)
    fin = np.where(np.isnan(flat), np.inf, flat)
    np.testing.assert_array_equal(mt.emin, fin.min(axis=1))
    fin = np.where(np.isnan(flat), -np.inf, flat)
    np.testing.assert_array_equal(mt.emax, fin.max(axis=1))


def test_plan_format_matches_one_shot(tmp_path, gpu_ctx):
    path = next(p for p in GOLDEN if p.stem == "types14_600")
    _, job, prob = load_golden(path, tmp_path)
    job.close()
    one = gpu_ctx.compute_text(prob).tobytes()
    plan = gpu_ctx.plan(prob)
    plan.run()
    mt = plan.format()
    assert mt.tobytes() == one
    plan.close()


def test_cli_device_writer_matches_host_writer(tmp_path, built):
    cli = ROOT / "autogrid_b200" / "_build" / "autogrid4_b200"
    path = next(p for p in GOLDEN if p.stem == "distance_maps")
    z = np.load(path, allow_pickle=False)
    outs = []
    for name, extra in (("dev", []), ("host", ["--host-writer"])):
        d = tmp_path / name
        d.mkdir()
        (d / "g.gpf").write_text(str(z["gpf"]))
        (d / "g.pdbqt").write_text(str(z["pdbqt"]))
        r = subprocess.run([str(cli), "-p", "g.gpf", "-l", "g.glg", *extra], cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        outs.append(d)
    fa, fb = _map_files(outs[0]), _map_files(outs[1])
    assert [p.name for p in fa] == [p.name for p in fb] and len(fa) >= 3
    for a, b in zip(fa, fb):
        assert a.read_bytes() == b.read_bytes(), a.name
    assert _extrema_table(outs[0] / "g.glg") == _extrema_table(outs[1] / "g.glg")
