"""Seeded synthetic receptors and GPFs with the shapes of the benchmark workloads.

No public dataset exists for this path; receptors are generated the same way
for every workload:
  * atoms uniform in a sphere of radius R (R = 45 * (N/10000)^(1/3) A unless
    given), heavy atoms at least 1.1 A apart (rejection sampling);
  * types C 45% / A 10% / N 10% / NA 3% / OA 15% / SA 2% / HD 15%;
  * every HD sits 1.0 A from a random N or OA parent (exempt from the spacing
    check against that parent only) and is written right after it, so the
    reference's +-20-atom bond scan (main.cpp:2309-2310) finds the bond;
  * charges N(0, 0.25) shifted to net zero, written %6.3f (PDBQT columns 71-76);
  * GPF: smooth 0.5, dielectric -0.1465, receptor_types in first-appearance
    order, receptor before gridcenter, gridcenter at the sphere centre.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HEAVY_TYPES = ["C", "A", "N", "NA", "OA", "SA"]
HEAVY_FRACS = [0.45, 0.10, 0.10, 0.03, 0.15, 0.02]  # of all atoms; HD takes the remaining 0.15
HD_FRAC = 0.15

LIGAND_TYPES_8 = ["A", "C", "HD", "N", "NA", "OA"]  # + e + d = 8 maps
LIGAND_TYPES_14 = ["A", "C", "HD", "N", "NA", "OA", "SA", "S", "P", "F", "Cl", "Br", "I", "Fe"]


@dataclass
class Receptor:
    coords: np.ndarray   # [N,3] absolute coordinates (A)
    types: list
    charges: np.ndarray  # [N]
    center: tuple

    def pdbqt(self) -> str:
        out = []
        for i, (xyz, t, q) in enumerate(zip(self.coords, self.types, self.charges)):
            name = (t if len(t) == 2 else t + "1")[:4]
            out.append("ATOM  %5d %-4s %3s %1s%4d    %8.3f%8.3f%8.3f%6.2f%6.2f    %6.3f %-2s\n"
                       % (i % 100000, name, "SYN", "A", (i // 10) % 10000, xyz[0], xyz[1], xyz[2],
                          1.0, 0.0, q, t))
        return "".join(out)


def _grid_key(p, cell):
    return tuple(np.floor(p / cell).astype(int))


def make_receptor(n_atoms: int, seed: int, radius: float | None = None,
                  center=(0.0, 0.0, 0.0), min_sep: float = 1.1) -> Receptor:
    """Generate a receptor of n_atoms atoms (see module docstring)."""
    rng = np.random.default_rng(seed)
    if radius is None:
        radius = 45.0 * (n_atoms / 10000.0) ** (1.0 / 3.0)
    n_hd = int(round(HD_FRAC * n_atoms))
    n_heavy = n_atoms - n_hd
    # heavy-atom types in proportion
    fr = np.array(HEAVY_FRACS) / sum(HEAVY_FRACS)
    counts = np.floor(fr * n_heavy).astype(int)
    counts[0] += n_heavy - counts.sum()
    htypes = np.repeat(np.arange(len(HEAVY_TYPES)), counts)
    rng.shuffle(htypes)

    cell = min_sep
    occupied: dict = {}
    pos = np.zeros((n_atoms, 3))

    def ok(p, exempt=-1):
        k = _grid_key(p, cell)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for j in occupied.get((k[0] + dx, k[1] + dy, k[2] + dz), ()):
                        if j != exempt and np.sum((pos[j] - p) ** 2) < min_sep * min_sep:
                            return False
        return True

    def put(i, p):
        pos[i] = p
        occupied.setdefault(_grid_key(p, cell), []).append(i)

    for i in range(n_heavy):
        for _ in range(10000):
            v = rng.uniform(-radius, radius, 3)
            if v @ v <= radius * radius and ok(v):
                put(i, v)
                break
        else:
            raise RuntimeError("could not place atom; density too high")
    parents_pool = [i for i in range(n_heavy) if HEAVY_TYPES[htypes[i]] in ("N", "OA")]
    children: dict = {}
    for k in range(n_hd):
        i = n_heavy + k
        for _ in range(10000):
            par = parents_pool[rng.integers(len(parents_pool))]
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            v = pos[par] + 1.0 * d
            if ok(v, exempt=par):
                put(i, v)
                children.setdefault(par, []).append(i)
                break
        else:
            raise RuntimeError("could not place HD atom")
    # file order: each heavy atom followed by its hydrogens
    order = []
    for i in range(n_heavy):
        order.append(i)
        order.extend(children.get(i, []))
    types_all = [HEAVY_TYPES[htypes[i]] for i in range(n_heavy)] + ["HD"] * n_hd
    q = rng.normal(0.0, 0.25, n_atoms)
    q -= q.mean()
    c = np.asarray(center, dtype=float)
    return Receptor(coords=pos[order] + c, types=[types_all[i] for i in order], charges=q[order],
                    center=tuple(c))


@dataclass
class GridSpec:
    npts: tuple = (40, 40, 40)
    spacing: float = 0.375
    ligand_types: list = field(default_factory=lambda: list(LIGAND_TYPES_8))
    elecmap: bool = True
    dsolvmap: bool = True
    dielectric: float = -0.1465
    smooth: float = 0.5
    extra_lines: list = field(default_factory=list)   # inserted after smooth
    pre_lines: list = field(default_factory=list)     # inserted before ligand_types
    center: tuple | None = None


def make_gpf(rec: Receptor, spec: GridSpec, stem: str) -> str:
    seen = []
    for t in rec.types:
        if t not in seen:
            seen.append(t)
    c = spec.center if spec.center is not None else rec.center
    lines = [f"npts {spec.npts[0]} {spec.npts[1]} {spec.npts[2]}",
             f"gridfld {stem}.maps.fld",
             f"spacing {spec.spacing}",
             "receptor_types " + " ".join(seen)]
    lines += list(spec.pre_lines)
    lines += ["ligand_types " + " ".join(spec.ligand_types),
              f"receptor {stem}.pdbqt",
              f"gridcenter {c[0]:.3f} {c[1]:.3f} {c[2]:.3f}",
              f"smooth {spec.smooth}"]
    lines += list(spec.extra_lines)
    for t in spec.ligand_types:
        lines.append(f"map {stem}.{t}.map")
        if "separate_desolvation_maps" in spec.pre_lines and t != "Z":
            lines.append(f"map {stem}.{t}.desolv.map")
    if spec.elecmap:
        lines.append(f"elecmap {stem}.e.map")
    if spec.dsolvmap:
        lines.append(f"dsolvmap {stem}.d.map")
    lines.append(f"dielectric {spec.dielectric}")
    return "\n".join(lines) + "\n"


def write_case(directory: str | Path, stem: str, rec: Receptor, spec: GridSpec) -> Path:
    """Write <stem>.pdbqt and <stem>.gpf into directory; returns the GPF path."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    (d / f"{stem}.pdbqt").write_text(rec.pdbqt())
    g = d / f"{stem}.gpf"
    g.write_text(make_gpf(rec, spec, stem))
    return g


# The benchmark workloads (sizes from the project's headline configurations).
WORKLOADS = {
    # 1,800 atoms in a 28 A sphere, npts 40^3 (41^3 points), 8 maps
    "ad4_1800_41cube_8maps": dict(n_atoms=1800, radius=28.0, spec=GridSpec(npts=(40, 40, 40))),
    # 10,000 atoms in a 45 A sphere, npts 126^3 (127^3 points), 14 types + e + d = 16 maps
    "ad4_10000_127cube_16maps": dict(n_atoms=10000, radius=45.0,
                                     spec=GridSpec(npts=(126, 126, 126), ligand_types=list(LIGAND_TYPES_14))),
    # the same receptor and maps on 49 of the 127 planes (a profiling case:
    # ~0.2 GB on the device, above the L2's 126 MB, one launch per kernel)
    "ad4_10000_127x127x49_16maps": dict(n_atoms=10000, radius=45.0,
                                        spec=GridSpec(npts=(126, 126, 48), ligand_types=list(LIGAND_TYPES_14))),
}


def workload(name: str, seed: int = 0) -> tuple:
    w = WORKLOADS[name]
    rec = make_receptor(w["n_atoms"], seed=seed, radius=w["radius"], center=(11.125, -4.5, 7.25))
    return rec, w["spec"]


# ----------------------------------------------------------------- ensembles --
ENSEMBLE_LIGANDS = list(LIGAND_TYPES_8)


def ensemble_specs(n: int, seed: int, atoms_range=(1000, 12000), npts_range=(20, 100)) -> list:
    """(n_atoms, npts) of each instance of a batched ensemble: atom counts
    log-uniform over atoms_range, per-axis npts uniform over npts_range
    (independently per axis; odd values are truncated to even by the GPF
    reader, as check_size.cpp:79-83 does)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(atoms_range[0]), np.log(atoms_range[1])
    out = []
    for _ in range(n):
        na = int(round(float(np.exp(rng.uniform(lo, hi)))))
        npts = tuple(int(v) for v in rng.integers(npts_range[0], npts_range[1] + 1, 3))
        out.append((na, npts))
    return out


def _write_instance(args):
    directory, i, na, npts, seed = args
    rec = make_receptor(na, seed=seed, center=(0.0, 0.0, 0.0))
    spec = GridSpec(npts=npts, ligand_types=list(ENSEMBLE_LIGANDS))
    return str(write_case(directory, f"inst{i:04d}", rec, spec))


def write_ensemble(directory, n: int, seed: int = 0, workers: int | None = None, **kw) -> list:
    """Write n instances (PDBQT + GPF) in parallel; returns the GPF paths."""
    import multiprocessing as mp
    import os
    specs = ensemble_specs(n, seed, **kw)
    jobs = [(str(directory), i, na, npts, seed * 100003 + i) for i, (na, npts) in enumerate(specs)]
    workers = workers or min(16, os.cpu_count() or 1)
    if workers <= 1 or n < 4:
        return [_write_instance(j) for j in jobs]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_write_instance, jobs)
