import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# the reference sources (tests that read them skip when they are absent)
from oracle.oracle import REFERENCE_SRC as REFERENCE  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Native library and oracle, built in-tree once per session."""
    from autogrid_b200 import build as agb_build
    from oracle import oracle as orc
    agb_build.build()
    orc.build(ref=REFERENCE.exists())
    return True


@pytest.fixture(scope="session")
def gpu_ctx(built):
    from autogrid_b200 import Context
    ctx = Context(0)
    yield ctx
    ctx.close()


def tolerance_ok(got, ref, abs_tol=1e-3, rel_tol=1e-4):
    """The parity bar: |got-ref| <= max(abs_tol, rel_tol*|ref|) elementwise."""
    return np.abs(got - ref) <= np.maximum(abs_tol, rel_tol * np.abs(ref))


def make_case(tmp_path, stem, n_atoms, npts, seed=0, radius=None, center=(1.5, -2.25, 3.0), **spec_kw):
    """Write a seeded synthetic receptor + GPF into tmp_path and load it with the front end."""
    from autogrid_b200 import Job, synth
    rec = synth.make_receptor(n_atoms, seed=seed, radius=radius, center=center)
    spec = synth.GridSpec(npts=npts, **spec_kw)
    gpf = synth.write_case(tmp_path, stem, rec, spec)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        job = Job(gpf.name, f"{stem}.glg")
        prob = job.problem()
    finally:
        os.chdir(cwd)
    return job, prob


FUZZ_LIGANDS = ["A", "C", "HD", "N", "NA", "OA", "SA", "S", "F", "Cl"]


def fuzz_config(seed):
    """Seeded random problem configuration: receptor size and sphere radius, box
    shape, spacing, ligand-type subset, smoothing, dielectric, qasp, disorder_h,
    separate desolvation maps and a covalent map (keyword arguments of make_case,
    plus n_atoms, npts, seed and radius)."""
    rng = np.random.default_rng(1000 + seed)
    n_atoms = int(rng.integers(80, 1600))
    # the generator's density (0.0262 atoms/A^3) or up to 2x sparser
    radius = 45.0 * (n_atoms / 10000.0) ** (1.0 / 3.0) * float(rng.uniform(1.0, 1.26))
    npts = tuple(int(v) for v in rng.integers(2, 24, 3))
    spacing = float(rng.choice([0.2, 0.3, 0.375, 0.5, 0.8]))
    types = sorted(rng.choice(FUZZ_LIGANDS, int(rng.integers(1, 7)), replace=False).tolist(), key=FUZZ_LIGANDS.index)
    pre, extra = [], []
    if rng.random() < 0.4:
        pre.append("disorder_h")
    if rng.random() < 0.3:
        pre.append("separate_desolvation_maps")
    if rng.random() < 0.3:
        extra.append(f"qasp {rng.uniform(0.005, 0.02):.4f}")
    if rng.random() < 0.25:
        extra.append("covalentmap 1.5 1000.0 1.0 -1.5 2.0")
    kw = dict(n_atoms=n_atoms, npts=npts, seed=int(seed), radius=radius, spacing=spacing, ligand_types=types,
              smooth=float(rng.choice([0.0, 0.25, 0.5, 1.0])),
              dielectric=float(rng.choice([-0.1465, -0.1465, 4.0, 40.0])),
              elecmap=bool(rng.random() < 0.85), dsolvmap=bool(rng.random() < 0.85),
              pre_lines=pre, extra_lines=extra)
    return kw
