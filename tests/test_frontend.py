"""Front end (ag_job_load): GPF keywords, receptor reader, fatal-error
behaviour and the .fld/.xyz/map-header writers, against the reference.

The pass/fail table is the reference test-suite's (Tests/test_autogrid4.py:341-389);
"success" here means the front end accepted the GPF (the GPU run is covered by
tests/test_gpu_cli.py).  x1hpv_CASE5 ("one map line too many") makes the
reference write past its gridmap[] array and crash (rc 139, main.cpp:1228,
:1513); this engine reports it as a fatal input error instead.
"""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REFERENCE, ROOT

needs_reference = pytest.mark.skipif(not (REFERENCE / "Tests").exists(), reason="reference sources absent")

FIXTURES = [
    ("x1hpv_CASE0", True), ("x1hpv_CASE1", False), ("x1hpv_CASE2", True), ("x1hpv_CASE3", True),
    ("x1hpv_CASE4", True), ("x1hpv_CASE5", False), ("hsg1_sm_nbpreps", True),
    ("hsg1_sm_nbpreps_illegal_atom", True), ("hsg1_sm_nbpreps_toofew", False), ("hsg1_sm_nbpcoeffs", True),
    ("hsg1_sm_no_parameter_file", True), ("hsg1_no_receptor_types", True), ("hsg1_sm", True),
    ("hsg1_sm_minus_two_types", False),
]


def _copy_tests(dst):
    for f in (REFERENCE / "Tests").iterdir():
        if f.suffix in (".gpf", ".pdbqt", ".dat"):
            shutil.copy(f, dst / f.name)


def _load(tmp_path, gpf, glg="out.glg"):
    from autogrid_b200 import AutoGridError, Job
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        try:
            return Job(gpf, glg), None
        except AutoGridError as e:
            return None, e
    finally:
        os.chdir(cwd)


@needs_reference
@pytest.mark.parametrize("stem,expect_ok", FIXTURES)
def test_reference_fixture_outcomes(stem, expect_ok, tmp_path, built):
    _copy_tests(tmp_path)
    job, err = _load(tmp_path, f"{stem}.gpf")
    assert (job is not None) == expect_ok, err
    glg = (tmp_path / "out.glg").read_text()
    if not expect_ok:
        assert "Unsuccessful Completion" in glg.splitlines()[-1] or "Unsuccessful Completion" in glg


@needs_reference
def test_fld_xyz_and_map_headers_match_reference(tmp_path, built):
    from oracle.oracle import REF_BIN
    mine, ref = tmp_path / "mine", tmp_path / "ref"
    mine.mkdir()
    ref.mkdir()
    _copy_tests(mine)
    _copy_tests(ref)
    subprocess.run([str(REF_BIN), "-p", "x1hpv_CASE0.gpf", "-l", "r.glg"], cwd=ref, check=True,
                   capture_output=True)
    job, err = _load(mine, "x1hpv_CASE0.gpf")
    assert job is not None, err
    prob = job.problem()
    job.write_maps(np.zeros(prob.map_shape, dtype=np.float64))
    drop = ("# Created by",)
    a = [ln for ln in (mine / "x1hpv.maps.fld").read_text().splitlines() if not ln.startswith(drop)]
    b = [ln for ln in (ref / "x1hpv.maps.fld").read_text().splitlines() if not ln.startswith(drop)]
    assert a == b
    assert (mine / "x1hpv.maps.xyz").read_text() == (ref / "x1hpv.maps.xyz").read_text()
    for name in ("A", "HD", "e", "d"):
        ha = (mine / f"x1hpv.{name}.map").read_text().splitlines()[:6]
        hb = (ref / f"x1hpv.{name}.map").read_text().splitlines()[:6]
        assert ha == hb


def test_map_writer_formatting(tmp_path, built):
    """Values below 1e-4 print as "0", others as %.3f of round3dp (main.cpp:3481-3496)."""
    from conftest import make_case
    job, prob = make_case(tmp_path, "w", 120, (2, 2, 2), seed=3, radius=7.0)
    vals = np.array([0.0, 5e-5, -9.9e-5, 1e-4, 0.0005, -0.0005, 1.2345, -1.2345, 99999.9996, 0.0015], dtype=np.float64)
    maps = np.zeros(prob.map_shape, dtype=np.float64).reshape(prob.n_maps, -1)
    maps[0, :vals.size] = vals
    job.write_maps(maps)
    lines = (tmp_path / "w.A.map").read_text().splitlines()[6:]
    expect = ["0", "0", "0", "0.000", "0.001", "-0.001", "1.234", "-1.234", "100000.000", "0.002"]
    assert lines[:vals.size] == expect


FATAL_GPFS = {
    "missing gridfld": ["npts 4 4 4", "spacing 0.375", "ligand_types C", "receptor r.pdbqt", "map r.C.map"],
    "elecmap before atom maps": ["npts 4 4 4", "gridfld r.maps.fld", "ligand_types C HD",
                                 "receptor r.pdbqt", "gridcenter 0 0 0", "map r.C.map", "elecmap r.e.map"],
    "too few maps": ["npts 4 4 4", "gridfld r.maps.fld", "ligand_types C HD", "receptor r.pdbqt",
                     "gridcenter 0 0 0", "map r.C.map"],
    "unknown ligand type": ["npts 4 4 4", "gridfld r.maps.fld", "ligand_types C Qx"],
    "npts too large": ["npts 2000 4 4"],
    "vina": ["use_vina_potential"],
    "ligand types before npts": ["gridfld r.maps.fld", "ligand_types C"],
    "separate desolvation after types": ["npts 4 4 4", "gridfld r.maps.fld", "ligand_types C",
                                         "separate_desolvation_maps"],
    "gridcenter before gridfld": ["npts 4 4 4", "gridcenter 0 0 0"],
}


@pytest.mark.parametrize("name", sorted(FATAL_GPFS))
def test_fatal_conditions(name, tmp_path, built):
    from autogrid_b200 import synth
    rec = synth.make_receptor(60, seed=1, radius=6.0)
    (tmp_path / "r.pdbqt").write_text(rec.pdbqt())
    (tmp_path / "bad.gpf").write_text("\n".join(FATAL_GPFS[name]) + "\n")
    job, err = _load(tmp_path, "bad.gpf")
    assert job is None and err is not None
    assert "Unsuccessful Completion" in (tmp_path / "out.glg").read_text()


def test_receptor_type_count_mismatch(tmp_path, built):
    from autogrid_b200 import synth
    rec = synth.make_receptor(80, seed=2, radius=6.0)
    (tmp_path / "r.pdbqt").write_text(rec.pdbqt())
    (tmp_path / "g.gpf").write_text("npts 4 4 4\ngridfld r.maps.fld\nreceptor_types C A\n"
                                    "ligand_types C\nreceptor r.pdbqt\n")
    job, err = _load(tmp_path, "g.gpf")
    assert job is None and "does not match" in err.message


def test_problem_layout_and_tables(tmp_path, built):
    """Spot-check the front end's tables against closed forms of main.cpp:1614-1627 and :2272-2276."""
    from conftest import make_case
    _, prob = make_case(tmp_path, "t", 150, (4, 4, 4), seed=4, radius=8.0)
    a = prob.arrays
    r = np.arange(8192) / 128.0
    sol = 0.1322 * np.exp(-(r * r) / (2 * 3.6 * 3.6))
    sol[0] = 0.0
    assert np.allclose(a["sol_fn"], sol, rtol=1e-15, atol=0)
    lam, eps0, A, rk = 0.003627, 78.4, -8.5525, 7.7839
    B = eps0 - A
    eps = A + B / (1.0 + rk * np.exp(-lam * B * r))
    eps[0] = 1.0
    assert np.allclose(a["r_epsilon_fn"], 332.0 / eps, rtol=1e-13)
    nt, nm = prob.scalars["n_rec_types"], prob.scalars["n_atom_maps"]
    tab = a["e_vdw_hb"].reshape(nt, nm, 1024)
    assert np.all(tab[:, :, 0] == 100000.0)
    assert prob.n_maps == nm + 2 and prob.scalars["elec_map"] == nm and prob.scalars["dsolv_map"] == nm + 1
