"""Generate the golden fixtures in tests/golden/*.npz from the reference itself.

Each fixture is a small seeded synthetic receptor + GPF (written by
autogrid_b200.synth) run through oracle/_ref/autogrid4_fullprec -- the
reference's own sources, compiled unmodified except that map values are
printed float-exact instead of %.3f (oracle/ref_fullprec_shim.h) -- and
oracle/_ref/autogrid4 (unmodified, %.3f output).  Stored per case: the GPF and
PDBQT text, the map names, the full-precision maps (float64 of the printed
float values), the %.3f maps, and the .fld text.

The collision fixtures (tests/golden/collision/*.npz) come from
oracle/_ref/autogrid4_bhtree_fullprec, the same sources built with the
reference's USE_BHTREE switch: the only build in which
'map_receptor_interior off' (collision points) exists.  Its LOOP 2 uses the
BH tree's single-precision distances, so only its e map, floating grid and
constriction grid are pinned exactly; the other maps are stored for the
parity bar.

Run here, where the reference sources exist:
    python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from autogrid_b200 import synth  # noqa: E402
from oracle import oracle as orc  # noqa: E402

OUT = Path(__file__).resolve().parent

CASES = {
    # default AD4.1 options, distance-dependent dielectric, 6 ligand types + e + d
    "basic_400": dict(n=400, seed=11, radius=11.0, spec=dict(npts=(10, 12, 14))),
    # every config-1 ligand type (halogens, Fe, P, S, SA)
    "types14_600": dict(n=600, seed=12, radius=13.0,
                        spec=dict(npts=(8, 8, 10), ligand_types=list(synth.LIGAND_TYPES_14))),
    # disorder_h, separate desolvation maps and a covalent map
    "disorder_sep_cov": dict(n=400, seed=13, radius=11.0, spec=dict(
        npts=(8, 10, 6), ligand_types=["A", "C", "HD", "OA", "NA", "Z"],
        pre_lines=["separate_desolvation_maps", "disorder_h"],
        extra_lines=["covalentmap 1.5 1000.0 1.0 -1.5 2.0"])),
    # constant dielectric, pairwise overrides, qasp/coefficient/smoothing changes
    "constdiel_nbp": dict(n=300, seed=14, radius=10.0, spec=dict(
        npts=(6, 6, 6), dielectric=4.0, smooth=0.25,
        extra_lines=["qasp 0.012", "nbp_r_eps 1.9 5.0 12 10 HD OA", "nbp_coeffs 1297.46 227.81 12 6 C A"])),
    # no e map, odd npts (truncated to even), coarser spacing
    "noelec_odd": dict(n=300, seed=15, radius=10.0, spec=dict(
        npts=(9, 11, 7), spacing=0.5, elecmap=False)),
    # one ligand map and no d map; a single grid point
    "tiny_onepoint": dict(n=200, seed=16, radius=8.0, spec=dict(
        npts=(1, 1, 1), ligand_types=["OA"], dsolvmap=False)),
    # floating grid and constriction grid (main.cpp:2947-2966, :3498-3514)
    "distance_maps": dict(n=300, seed=17, radius=10.0, dist=["f", "c"], spec=dict(
        npts=(10, 8, 12), ligand_types=["C", "OA"],
        extra_lines=["fmap g.f.map", "constriction_distance_cutoff 5.5", "cmap g.c.map"])),
}


COLLISION_CASES = {
    # map_receptor_interior off: e = 0 and fmap = 1.5 within 1.5 A of an atom,
    # the BH tree's constriction count (main.cpp:2893-2927)
    "bhtree_collision": dict(n=300, seed=18, radius=9.0, spec=dict(
        npts=(10, 12, 8), ligand_types=["A", "C", "HD", "OA"],
        extra_lines=["map_receptor_interior off", "fmap g.f.map", "constriction_distance_cutoff 5.5",
                     "cmap g.c.map"])),
    # the same without distance maps, constant dielectric, a denser receptor
    "bhtree_collision_constdiel": dict(n=500, seed=19, radius=9.0, spec=dict(
        npts=(8, 8, 10), dielectric=10.0, ligand_types=["C", "NA"], extra_lines=["map_receptor_interior off"])),
}


def map_names(spec: synth.GridSpec) -> list:
    names = []
    for t in spec.ligand_types:
        names.append(t)
        if "separate_desolvation_maps" in spec.pre_lines and t != "Z":
            names.append(t + ".desolv")
    if spec.elecmap:
        names.append("e")
    if spec.dsolvmap:
        names.append("d")
    return names


def run_reference(binary: Path, d: Path, stem: str) -> None:
    r = subprocess.run([str(binary), "-p", f"{stem}.gpf", "-l", f"{stem}.glg"], cwd=d,
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed on {stem}: {r.stderr[-500:]}")


def make(name: str, case: dict) -> Path:
    rec = synth.make_receptor(case["n"], seed=case["seed"], radius=case["radius"], center=(2.125, -1.5, 0.75))
    spec = synth.GridSpec(**case["spec"])
    names = map_names(spec)
    full, rounded = [], []
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        gpf = synth.write_case(d, "g", rec, spec)
        dist = case.get("dist", [])
        run_reference(orc.REF_FULLPREC_BIN, d, "g")
        full = [orc.read_map(d / f"g.{n}.map") for n in names]
        dist_full = [orc.read_map(d / f"g.{n}.map") for n in dist]
        fld = (d / "g.maps.fld").read_text()
        run_reference(orc.REF_BIN, d, "g")
        rounded = [orc.read_map(d / f"g.{n}.map") for n in names]
        dist_3dp = [orc.read_map(d / f"g.{n}.map") for n in dist]
        out = OUT / f"{name}.npz"
        extra = {}
        if dist:
            extra = dict(dist_names=np.array(dist), dist_full=np.array(dist_full), dist_3dp=np.array(dist_3dp))
        np.savez_compressed(out, gpf=gpf.read_text(), pdbqt=(d / "g.pdbqt").read_text(),
                            names=np.array(names), maps_full=np.array(full), maps_3dp=np.array(rounded),
                            fld=fld, npts=np.array(spec.npts), **extra)
    return out


def make_collision(name: str, case: dict) -> Path:
    rec = synth.make_receptor(case["n"], seed=case["seed"], radius=case["radius"], center=(2.125, -1.5, 0.75))
    spec = synth.GridSpec(**case["spec"])
    names = map_names(spec)
    dist = [n for n, line in (("f", "fmap"), ("c", "cmap")) if any(x.startswith(line) for x in spec.extra_lines)]
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        gpf = synth.write_case(d, "g", rec, spec)
        run_reference(orc.REF_BHTREE_BIN, d, "g")
        full = [orc.read_map(d / f"g.{n}.map") for n in names]
        dist_full = [orc.read_map(d / f"g.{n}.map") for n in dist]
        (OUT / "collision").mkdir(exist_ok=True)
        out = OUT / "collision" / f"{name}.npz"
        np.savez_compressed(out, gpf=gpf.read_text(), pdbqt=(d / "g.pdbqt").read_text(), names=np.array(names),
                            maps_full=np.array(full), dist_names=np.array(dist),
                            dist_full=np.array(dist_full) if dist else np.zeros((0, 0)), npts=np.array(spec.npts))
    return out


def main():
    orc.build(ref=True)
    only = sys.argv[1:]
    for name, case in CASES.items():
        if only and name not in only:
            continue
        p = make(name, case)
        print(f"{p.name}: {p.stat().st_size} bytes")
    for name, case in COLLISION_CASES.items():
        if only and name not in only:
            continue
        p = make_collision(name, case)
        print(f"collision/{p.name}: {p.stat().st_size} bytes")


if __name__ == "__main__":
    main()
