"""Pin the FP64 oracle (oracle/ag_oracle.c) -- together with the C++ front end
that builds its input -- against the reference itself:

  * tests/golden/*.npz: maps the reference's own build printed at full float
    precision (tests/golden/make_golden.py) for seeded synthetic cases covering
    disorder_h, separate desolvation maps, a covalent map, constant dielectric,
    nbp_r_eps / nbp_coeffs overrides, odd npts and a single-point grid;
  * the reference test-suite's golden maps Tests/py_hsg1_sm.*.map, with the
    reference's own comparison rule (test_autogrid4.py:157-186);
  * live runs of oracle/_ref/autogrid4_fullprec on the reference's test inputs
    and on seeded random configurations (conftest.fuzz_config).
"""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REFERENCE, ROOT, fuzz_config

GOLDEN = sorted((ROOT / "tests" / "golden").glob("*.npz"))


def load_golden(path, tmp_path):
    """Recreate a golden case's files and load them with the front end."""
    from autogrid_b200 import Job
    z = np.load(path, allow_pickle=False)
    (tmp_path / "g.gpf").write_text(str(z["gpf"]))
    (tmp_path / "g.pdbqt").write_text(str(z["pdbqt"]))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        job = Job("g.gpf", "g.glg")
        prob = job.problem()
    finally:
        os.chdir(cwd)
    return z, job, prob


def full_precision_ok(got, ref):
    """Reference values were printed as floats (%.9g); values below 1e-4 as '0'."""
    tol = np.where(ref == 0.0, 1e-4, 1.5e-7 * np.abs(ref) + 1e-12)
    return np.abs(got - ref) <= tol


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_golden(path, tmp_path, built):
    from oracle.oracle import oracle_points
    z, job, prob = load_golden(path, tmp_path)
    ref = z["maps_full"]
    assert prob.n_maps == ref.shape[0]
    got, flags = oracle_points(prob)
    ok = full_precision_ok(got, ref)
    bad = np.argwhere(~ok)
    assert bad.size == 0, f"{len(bad)} values differ, first {bad[:3].tolist()}"
    if "dist_full" in z.files:  # floating grid (Angstrom, printed like a map) and constriction counts
        from oracle.oracle import oracle_distance_maps
        dist = oracle_distance_maps(prob)
        assert dist.shape == z["dist_full"].shape
        assert np.all(np.abs(dist[0] - z["dist_full"][0]) <= 1.5e-7 * np.abs(z["dist_full"][0]))
        assert np.array_equal(dist[1], z["dist_full"][1])


def test_golden_set_is_present():
    assert len(GOLDEN) >= 6


needs_reference = pytest.mark.skipif(not (REFERENCE / "Tests").exists(), reason="reference sources absent")


def _copy_tests(tmp_path):
    for f in (REFERENCE / "Tests").iterdir():
        if f.suffix in (".gpf", ".pdbqt", ".dat"):
            shutil.copy(f, tmp_path / f.name)


@needs_reference
def test_oracle_vs_reference_testsuite_golden_maps(tmp_path, built):
    """Tests/py_hsg1_sm.*.map with the rule of test_autogrid4.py:157-186, bounded
    by the reference's own deviation from those maps (max 0.003 kcal/mol)."""
    from autogrid_b200 import Job
    from oracle.oracle import oracle_points, read_map
    _copy_tests(tmp_path)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        prob = Job("hsg1_sm.gpf", "hsg1_sm.glg").problem()
    finally:
        os.chdir(cwd)
    got, _ = oracle_points(prob)
    for i, name in enumerate(["A", "C", "HD", "N", "NA", "OA", "e", "d"]):
        py = read_map(REFERENCE / "Tests" / f"py_hsg1_sm.{name}.map")
        mine = np.round(got[i], 3)
        assert np.abs(mine - py).max() <= 0.0035, name


@needs_reference
@pytest.mark.parametrize("stem", ["hsg1_sm", "x1hpv_CASE0", "hsg1_sm_nbpreps", "hsg1_sm_nbpcoeffs",
                                  "hsg1_sm_no_parameter_file", "hsg1_no_receptor_types"])
def test_oracle_vs_live_reference(stem, tmp_path, built):
    from autogrid_b200 import Job
    from oracle.oracle import REF_FULLPREC_BIN, oracle_points, read_map
    _copy_tests(tmp_path)
    ref_dir = tmp_path / "ref"
    ref_dir.mkdir()
    _copy_tests(ref_dir)
    r = subprocess.run([str(REF_FULLPREC_BIN), "-p", f"{stem}.gpf", "-l", f"{stem}.glg"], cwd=ref_dir,
                       capture_output=True, text=True)
    assert r.returncode == 0
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        job = Job(f"{stem}.gpf", f"{stem}.glg")
        prob = job.problem()
    finally:
        os.chdir(cwd)
    got, _ = oracle_points(prob)
    gpf = (tmp_path / f"{stem}.gpf").read_text().splitlines()
    files = [ln.split()[1] for ln in gpf if ln.split() and ln.split()[0] in ("map", "elecmap", "dsolvmap")]
    assert len(files) == prob.n_maps
    for i, f in enumerate(files):
        ref = read_map(ref_dir / f)
        ok = full_precision_ok(got[i], ref)
        assert ok.all(), f"{stem} {f}: max |d| {np.abs(got[i] - ref).max()}"


def _map_files(gpf_text):
    return [ln.split()[1] for ln in gpf_text.splitlines()
            if ln.split() and ln.split()[0] in ("map", "elecmap", "dsolvmap")]


@needs_reference
@pytest.mark.parametrize("seed", range(int(os.environ.get("AG_FUZZ_SEEDS", "12"))))
def test_oracle_vs_live_reference_random(seed, tmp_path, built):
    """The seeded random configurations of the GPU fuzz test through the
    reference's full-precision build: front end + oracle equal its maps at
    every point.  A configuration the reference rejects (a disorder_h bond
    overflow, bondmanager.cpp:44-88 via main.cpp:2396-2406) must be rejected by
    the front end with the same message; it is then drawn without disorder_h.
    AG_FUZZ_SEEDS sets the number of configurations (default 12; 64 pass)."""
    from autogrid_b200 import AutoGridError, Job, synth
    from oracle.oracle import REF_FULLPREC_BIN, oracle_points, read_map
    kw = fuzz_config(seed)
    rec = synth.make_receptor(kw.pop("n_atoms"), seed=kw.pop("seed"), radius=kw.pop("radius"),
                              center=(1.5, -2.25, 3.0))
    npts = kw.pop("npts")

    def run(stem):
        spec = synth.GridSpec(npts=npts, **kw)
        ref_dir, own_dir = tmp_path / f"{stem}_ref", tmp_path / f"{stem}_own"
        synth.write_case(ref_dir, stem, rec, spec)
        synth.write_case(own_dir, stem, rec, spec)
        r = subprocess.run([str(REF_FULLPREC_BIN), "-p", f"{stem}.gpf", "-l", f"{stem}.glg"], cwd=ref_dir,
                           capture_output=True, text=True)
        cwd = os.getcwd()
        os.chdir(own_dir)
        try:
            prob, err = Job(f"{stem}.gpf", f"{stem}.glg").problem(), None
        except AutoGridError as e:
            prob, err = None, e
        finally:
            os.chdir(cwd)
        return ref_dir, r, prob, err

    ref_dir, r, prob, err = run("f")
    if r.returncode != 0:
        said = r.stdout + r.stderr + (ref_dir / "f.glg").read_text(errors="replace")
        assert "could not add bond" in said, said[-400:]
        assert err is not None and "could not add bond" in err.message
        kw["pre_lines"] = [ln for ln in kw["pre_lines"] if ln != "disorder_h"]
        ref_dir, r, prob, err = run("g")
    assert r.returncode == 0 and err is None, (r.stderr[-400:], err)
    got, _ = oracle_points(prob)
    files = _map_files(next(ref_dir.glob("*.gpf")).read_text())
    assert len(files) == prob.n_maps
    for i, f in enumerate(files):
        ref = read_map(ref_dir / f)
        ok = full_precision_ok(got[i], ref)
        assert ok.all(), f"seed {seed} {f}: {int((~ok).sum())} values off, max |d| {np.abs(got[i] - ref).max()}"


COLLISION = sorted((ROOT / "tests" / "golden" / "collision").glob("*.npz"))


def _collision_check(prob, z):
    """The oracle against the USE_BHTREE reference: e map, floating and
    constriction grids exactly (the printed float precision), the LOOP 2 maps
    within the parity bar (that build's LOOP 2 takes the BH tree's
    single-precision distances)."""
    from conftest import tolerance_ok
    from oracle.oracle import oracle_distance_maps, oracle_points
    o, _ = oracle_points(prob)
    ref = z["maps_full"]
    names = [str(n) for n in z["names"]]
    for k, n in enumerate(names):
        if n == "e":
            assert full_precision_ok(o[k][None], ref[k][None]).all()
        else:
            assert tolerance_ok(o[k], ref[k]).all(), n
    e = names.index("e") if "e" in names else None
    if e is not None:
        assert (o[e] == 0.0).sum() == (ref[e] == 0.0).sum() > 0  # the collision points
    if z["dist_full"].size:
        dm = oracle_distance_maps(prob)
        assert np.all(np.abs(dm[0] - z["dist_full"][0]) <= 1.5e-7 * np.abs(z["dist_full"][0]))
        assert np.array_equal(dm[1], z["dist_full"][1])


@pytest.mark.parametrize("path", COLLISION, ids=[p.stem for p in COLLISION])
def test_oracle_collision_mode_matches_bhtree_reference(path, tmp_path, built):
    assert len(COLLISION) == 2
    z, job, prob = load_golden(path, tmp_path)
    assert prob.scalars["report_collisions"] == 1
    _collision_check(prob, z)


@needs_reference
@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_collision_mode_vs_live_bhtree(seed, tmp_path, built):
    """Random receptors with 'map_receptor_interior off' through the reference's
    USE_BHTREE build, live."""
    import subprocess
    from autogrid_b200 import Job, synth
    from oracle.oracle import REF_BHTREE_BIN, read_map
    rng = np.random.default_rng(700 + seed)
    rec = synth.make_receptor(int(rng.integers(150, 500)), seed=seed + 90, radius=float(rng.uniform(6.0, 10.0)))
    spec = synth.GridSpec(npts=tuple(int(v) for v in rng.integers(4, 14, 3)), spacing=float(rng.choice([0.3, 0.375, 0.5])),
                          ligand_types=["C", "OA", "HD"],
                          extra_lines=["map_receptor_interior off", "fmap g.f.map",
                                       f"constriction_distance_cutoff {rng.uniform(3.0, 7.9):.2f}", "cmap g.c.map"])
    synth.write_case(tmp_path, "g", rec, spec)
    r = subprocess.run([str(REF_BHTREE_BIN), "-p", "g.gpf", "-l", "g.glg"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    names = ["C", "OA", "HD", "e", "d"]
    z = {"names": np.array(names), "maps_full": np.array([read_map(tmp_path / f"g.{n}.map") for n in names]),
         "dist_full": np.array([read_map(tmp_path / "g.f.map"), read_map(tmp_path / "g.c.map")])}
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        prob = Job("g.gpf", "mine.glg").problem()
    finally:
        os.chdir(cwd)
    _collision_check(prob, z)
