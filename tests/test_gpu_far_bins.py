"""Far-field table bins: every far pair's bin equals the reference's.

The reference bins each LOOP 1 pair as (int)(A_DIV * r), r = hypot(dx,
hypot(dy, dz)) in double (main.cpp:97, :2951-2956).  The far-field kernel
computes distances in FP32; a pair whose FP32 distance lies within its error
bound of a bin edge is flagged and resolved in FP64.  These tests dump the
bin the kernel's arithmetic gives each (point, atom) pair (ag_diag_far_bins)
and compare it with the reference's expression evaluated here with the host
libm's hypot.  The only pairs allowed to differ are those whose reference
distance lies within 1e-12 of a bin edge (the contract's "within one ulp"
pairs), which are counted.
"""
import numpy as np
import pytest

from conftest import make_case
from test_oracle_pinning import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

NDIEL = 8192


def reference_bins(prob, pts):
    """(bin, tie) of the reference's LOOP 1 lookup for points x atoms."""
    coord = prob.arrays["coord"].reshape(-1, 3)
    n1, ne, sp = prob.n1, prob.ne, float(prob.scalars["spacing"])
    ix = pts % n1[0]
    iy = (pts // n1[0]) % n1[1]
    iz = pts // (n1[0] * n1[1])
    c = [(ix - ne[0]) * sp, (iy - ne[1]) * sp, (iz - ne[2]) * sp]  # main.cpp:2859
    d = [coord[None, :, k] - c[k][:, None] for k in range(3)]
    r = np.hypot(d[0], np.hypot(d[1], d[2]))
    r = np.maximum(r, 1e-6)
    t = r * 128.0
    tie = np.abs(t - np.rint(t)) <= 1e-12 * t
    return np.minimum(t.astype(np.int64), NDIEL - 1), tie


def check_bins(ctx, prob, pts, chunk=4096):
    totals = dict(owned=0, flagged=0, fp32_wrong=0, fp32_vs_used=0, ties=0, ref_ties=0)
    for k in range(0, len(pts), chunk):
        p = pts[k:k + chunk]
        used, fp32, flags = ctx.far_bins(prob, p)
        ref, tie = reference_bins(prob, p)
        owned = used >= 0
        flagged = (flags & 1) != 0
        # no unflagged pair may differ from the reference
        bad = owned & ~flagged & (used != ref)
        assert not bad.any(), f"{int(bad.sum())} unflagged far pairs with a wrong bin"
        # resolved pairs equal the reference except at FP64 ties
        bad = owned & (used != ref) & ~tie
        assert not bad.any(), f"{int(bad.sum())} far pairs with a wrong bin (not ties)"
        # every plain-FP32 bin error was caught by the guard
        wrong32 = owned & (np.minimum(fp32, NDIEL - 1) != ref)
        assert not (wrong32 & ~flagged).any()
        totals["owned"] += int(owned.sum())
        totals["flagged"] += int((owned & flagged).sum())
        totals["fp32_wrong"] += int(wrong32.sum())
        # the kernel's own count: resolved pairs whose plain FP32 bin is not the resolved one
        totals["fp32_vs_used"] += int((owned & flagged & (np.minimum(fp32, NDIEL - 1) != used)).sum())
        totals["ties"] += int((owned & ((flags & 2) != 0)).sum())
        totals["ref_ties"] += int((owned & tie).sum())
    return totals


def test_rsqrt_error_within_guard_assumption(gpu_ctx):
    """The guard's error bound takes rsqrt.approx.f32 at 2.5 * 2^-24 relative
    error over the squared distances the far kernel sees (bins^2 in [2^20, 2^27))."""
    import ctypes as C
    from autogrid_b200 import load_library
    v = C.c_double()
    assert load_library().ag_diag_rsqrt_error(0, 20, 28, C.byref(v)) == 0
    assert 0.0 < v.value <= 2.5, v.value


@pytest.mark.parametrize("name", ["basic_400", "types14_600"])
def test_golden_far_bins_exact(name, tmp_path, gpu_ctx):
    path = next(p for p in GOLDEN if p.stem == name)
    _, _, prob = load_golden(path, tmp_path)
    pts = np.arange(prob.points, dtype=np.int64)
    tot = check_bins(gpu_ctx, prob, pts)
    assert tot["owned"] > 0


def test_config0_far_bins_exact_and_counted(tmp_path, gpu_ctx):
    """1,800 atoms, 41^3 points, 0.375 A: every pair of the grid.  The guard's
    count equals the far kernel's own count in ag_stats, and plain FP32 bins
    would have been wrong for some pairs (so the guard is doing work)."""
    _, prob = make_case(tmp_path, "c0", 1800, (40, 40, 40), seed=3, radius=28.0, center=(0.0, 0.0, 0.0))
    pts = np.arange(prob.points, dtype=np.int64)
    tot = check_bins(gpu_ctx, prob, pts, chunk=2048)
    gpu_ctx.compute(prob, "fp32")
    st = gpu_ctx.stats()
    assert st.far_edge_pairs == tot["flagged"]
    assert st.far_fp32_bin_errors == tot["fp32_vs_used"]
    assert st.far_fp64_ties == tot["ties"]
    # the two differ only where a tie was decided by CUDA's hypot instead of the host's
    assert abs(tot["fp32_vs_used"] - tot["fp32_wrong"]) <= tot["ref_ties"]
    assert tot["fp32_wrong"] > 0
    assert tot["flagged"] < 0.01 * tot["owned"]


def test_spacing_with_inexact_frame_coordinates(tmp_path, gpu_ctx):
    """0.4 A spacing: frame point coordinates (multiples of 51.2 bins) are not
    exact floats, which widens the guard; the bins stay exact."""
    _, prob = make_case(tmp_path, "sp04", 900, (30, 24, 26), seed=5, spacing=0.4)
    rng = np.random.default_rng(1)
    pts = np.unique(rng.integers(0, prob.points, 3000)).astype(np.int64)
    tot = check_bins(gpu_ctx, prob, pts)
    assert tot["owned"] > 0


def test_clamped_far_table(tmp_path, gpu_ctx):
    """A 60 A receptor with the box near its edge: atom-point distances from a
    few A to ~135 A, beyond the longest extended far table (FAR_TAB_MAX bins,
    128 A), so the far kernel clamps t at the last bin, as the reference's
    min(lookup(r), NDIEL - 1) does.  Bins and the e map still match the
    reference expression and the oracle."""
    import os
    from conftest import tolerance_ok
    from autogrid_b200 import Job, synth
    from oracle.oracle import oracle_points
    rec = synth.make_receptor(700, seed=11, radius=60.0, center=(0.0, 0.0, 0.0))
    spec = synth.GridSpec(npts=(10, 12, 8), center=(76.0, 5.0, -3.0))
    gpf = synth.write_case(tmp_path, "clamp", rec, spec)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        prob = Job(gpf.name, None).problem()
    finally:
        os.chdir(cwd)
    coord = prob.arrays["coord"].reshape(-1, 3)  # relative to the grid centre
    dmax = float(np.max(np.linalg.norm(coord, axis=1)))
    assert dmax > 132.0  # the extended table would need more than FAR_TAB_MAX (16,384) bins
    pts = np.arange(prob.points, dtype=np.int64)
    tot = check_bins(gpu_ctx, prob, pts)
    assert tot["owned"] > 0 and tot["flagged"] > 0
    maps = gpu_ctx.compute(prob, "fp32").reshape(prob.n_maps, -1)
    ref, flags = oracle_points(prob)
    assert (tolerance_ok(maps, ref) | (flags[None, :] != 0)).all()
