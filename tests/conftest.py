import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

REFERENCE = Path(os.environ.get("AG_REFERENCE_SRC", "/root/reference"))


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
