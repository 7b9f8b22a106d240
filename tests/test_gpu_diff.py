"""Differentiable mode on the GPU (ag_diff_*, torch binding).

* forward: FP64 twin vs the FP64 C oracle's restatement of the linear-table
  mode (oracle/ag_oracle.c ag_oracle_points_lin) to 1e-9, the FP32 kernels to
  the drop-in parity bar; closest DS/D1 atoms vs the reference's search;
* adjoint: FP64 adjoint vs central differences of the FP64 forward
  (1e-4 e on charges; 1e-3 down to 1e-6 A on coordinates, closest hydrogens
  and bonded neighbours frozen), FP32 adjoint vs FP64 adjoint.  The tables
  are piecewise linear over bins of 1/128 A, so a coordinate step straddles
  slope kinks of the loss; each straddled kink adds a finite-difference error
  of fixed size and their number grows with h, so the agreement is asserted
  to tighten as h shrinks;
* the torch.autograd binding returns the same gradients as the C ABI.
"""
import numpy as np
import pytest

from conftest import make_case, tolerance_ok

pytestmark = pytest.mark.gpu

CASES = {
    "plain": dict(n_atoms=500, npts=(16, 16, 16), seed=3, radius=12.0),
    "disorder_sep": dict(n_atoms=500, npts=(14, 16, 12), seed=4, radius=12.0,
                         pre_lines=["disorder_h", "separate_desolvation_maps"]),
    "constdiel": dict(n_atoms=400, npts=(12, 12, 12), seed=5, radius=11.0, dielectric=40.0),
}


def _case(tmp_path, name):
    kw = dict(CASES[name])
    return make_case(tmp_path, name, kw.pop("n_atoms"), kw.pop("npts"), seed=kw.pop("seed"),
                     radius=kw.pop("radius"), **kw)


def _reference_closest_h(prob):
    """main.cpp:2986-3015: DS/D1 atoms in file order, strict <, FP64."""
    n1x, n1y, n1z = prob.n1
    nex, ney, nez = prob.ne
    sp = prob.scalars["spacing"]
    c = prob.arrays["coord"].reshape(-1, 3)
    hb = prob.arrays["hbond"]
    hidx = np.flatnonzero((hb == 1) | (hb == 2))
    iz, iy, ix = np.meshgrid(np.arange(n1z), np.arange(n1y), np.arange(n1x), indexing="ij")
    px = ((ix.ravel() - nex) * sp)[:, None]
    py = ((iy.ravel() - ney) * sp)[:, None]
    pz = ((iz.ravel() - nez) * sp)[:, None]
    d0 = c[hidx, 0][None, :] - px
    d1 = c[hidx, 1][None, :] - py
    d2 = c[hidx, 2][None, :] - pz
    r = np.sqrt(d0 * d0 + d1 * d1 + d2 * d2)
    return hidx[np.argmin(r, axis=1)].astype(np.int32)


@pytest.mark.parametrize("name", list(CASES))
def test_linear_forward_matches_oracle(tmp_path, gpu_ctx, name):
    from autogrid_b200 import Diff
    from oracle.oracle import oracle_points_lin
    _, prob = _case(tmp_path, name)
    d64 = Diff(gpu_ctx, prob, "fp64")
    d64.forward()
    ch = d64.closest_h()
    assert np.array_equal(ch, _reference_closest_h(prob))
    ref = oracle_points_lin(prob, closest_h=ch)
    got64 = d64.maps().reshape(prob.n_maps, -1)
    np.testing.assert_allclose(got64, ref, rtol=1e-9, atol=1e-9)
    d32 = Diff(gpu_ctx, prob, "fp32")
    d32.forward()
    assert np.array_equal(d32.closest_h(), ch)
    got32 = d32.maps().reshape(prob.n_maps, -1).astype(np.float64)
    ok = tolerance_ok(got32, ref)
    assert ok.all(), f"{(~ok).sum()} FP32 values off; worst {np.abs(got32 - ref).max()}"
    d32.close(); d64.close()


def test_linear_mode_agrees_with_nearest_bin_at_bin_resolution(tmp_path, gpu_ctx):
    """The interpolated maps stay within one table step of the drop-in maps."""
    from autogrid_b200 import Diff
    _, prob = _case(tmp_path, "plain")
    near = gpu_ctx.compute(prob, "fp64").reshape(prob.n_maps, -1)
    d = Diff(gpu_ctx, prob, "fp64")
    d.forward()
    lin = d.maps().reshape(prob.n_maps, -1)
    e = prob.scalars["elec_map"]
    # e map: the dielectric table changes by < 0.5% per bin beyond 0.5 A
    np.testing.assert_allclose(lin[e], near[e], rtol=2e-2, atol=5e-2)
    d.close()


@pytest.mark.parametrize("name", ["plain", "disorder_sep"])
def test_adjoint_matches_central_differences(tmp_path, gpu_ctx, name):
    from autogrid_b200 import gradcheck
    job, prob = _case(tmp_path, name)
    rng = np.random.default_rng(11)
    w = rng.normal(size=prob.map_shape)
    # atoms near the box, where every map term acts
    c = prob.arrays["coord"].reshape(-1, 3)
    half = np.array(prob.ne) * prob.scalars["spacing"]
    near_box = np.flatnonzero(np.all(np.abs(c) < half + 4.0, axis=1))
    atoms = rng.choice(near_box, 16, replace=False)
    hs = (1e-3, 1e-4, 1e-5, 1e-6)
    r = gradcheck.check(job, prob, gpu_ctx, atoms, w, h_coord=hs)
    err = r["fp64_vs_fd_coord"]
    print({h: f"{e:.3g}" for h, e in err.items()}, r["fp64_vs_fd_charge"], r["fp32_vs_fp64_coord"])
    assert r["fp64_vs_fd_charge"] < 1e-6, r["fp64_vs_fd_charge"]
    # table kinks every 1/128 A: the finite-difference error falls with h
    assert err[1e-6] < 1e-4, err
    assert err[1e-5] < 1e-3, err
    assert err[1e-3] < 2e-2, err
    assert r["fp32_vs_fp64_coord"] < 1e-3, r["fp32_vs_fp64_coord"]
    assert r["fp32_vs_fp64_charge"] < 1e-3, r["fp32_vs_fp64_charge"]


def test_torch_binding_matches_c_abi(tmp_path, gpu_ctx):
    import torch
    from autogrid_b200 import gradcheck
    from autogrid_b200.api import Diff
    from autogrid_b200.torch_maps import GridMaps
    job, prob = _case(tmp_path, "plain")
    fn = GridMaps(job, device=0, precision="fp64")
    coords = torch.tensor(prob.arrays["coord"].reshape(-1, 3), dtype=torch.float64, requires_grad=True)
    charges = torch.tensor(prob.arrays["charge"], dtype=torch.float64, requires_grad=True)
    maps = fn(coords, charges)
    assert maps.is_cuda and maps.shape == prob.map_shape
    w = torch.randn(prob.map_shape, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    (w * maps).sum().backward()
    d = Diff(gpu_ctx, prob, "fp64")
    d.forward()
    # the binding rebuilds the bond vectors on the device (CUDA hypot, FMA):
    # equal to the host's to the last bits
    m = d.maps()
    np.testing.assert_allclose(maps.detach().cpu().numpy(), m, rtol=1e-12, atol=1e-12 * np.abs(m).max())
    gc, gq = gradcheck.full_gradient(job, d, prob.arrays["coord"].reshape(-1, 3), w.cpu().numpy())
    np.testing.assert_allclose(coords.grad.numpy(), gc, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(charges.grad.numpy(), gq, rtol=1e-9, atol=1e-9)
    d.close()


def test_distance_maps_in_differentiable_mode(tmp_path, gpu_ctx):
    """fmap/cmap after the energy maps: equal to the drop-in path's (same FP64
    kernel); the floating grid's gradient (nearest atom's unit vector) matches
    central differences, the constriction grid contributes none."""
    from autogrid_b200 import Diff
    job, prob = make_case(tmp_path, "dm", 300, (10, 12, 8), seed=31, radius=9.0,
                          extra_lines=["fmap dm.f.map", "constriction_distance_cutoff 5.5", "cmap dm.c.map"])
    nm = prob.n_maps
    assert prob.n_out == nm + 2
    drop = gpu_ctx.compute(prob, "fp64").reshape(prob.n_out, -1)
    d = Diff(gpu_ctx, prob, "fp64")
    d.forward()
    got = d.maps().reshape(prob.n_out, -1)
    assert np.array_equal(got[nm:], drop[nm:])
    # gradient of L = sum w * fmap (energy and constriction weights zero)
    rng = np.random.default_rng(2)
    w = np.zeros(prob.map_shape)
    w[nm] = rng.normal(size=prob.map_shape[1:])
    gc = d.backward(w)["coord"]
    c0 = prob.arrays["coord"].reshape(-1, 3).copy()
    near = np.flatnonzero(np.abs(gc).sum(1) > 0)
    assert near.size > 0
    h = 1e-6
    for a in rng.choice(near, min(6, near.size), replace=False):
        for i in range(3):
            cp = c0.copy(); cp[a, i] += h
            cm = c0.copy(); cm[a, i] -= h
            d.set_atoms(cp); d.forward(keep_closest_h=True); lp = float(np.sum(w * d.maps()))
            d.set_atoms(cm); d.forward(keep_closest_h=True); lm = float(np.sum(w * d.maps()))
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gc[a, i]) <= 1e-5 * max(1.0, abs(gc[a, i])), (a, i, fd, gc[a, i])
    d.close()
