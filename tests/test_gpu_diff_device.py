"""Device-resident updates of the differentiable mode (ag_diff_set_bonds,
ag_diff_set_atoms_device, ag_diff_backward_device) against the host path
(coordinates, charges and bond vectors from ag_job_bond_vectors through
ag_diff_set_conformer; the bond-vector chain rule ag_job_bond_vectors_backward).

* maps of several jittered conformers agree with the host path to 1e-10
  (FP64 kernels) -- the device bond vectors (main.cpp:2297-2659 on the frozen
  topology) and cell lists reproduce the host's;
* the full coordinate gradient of the device adjoint (pair terms + bond-vector
  chain) equals the host's pair terms + host chain to 1e-9, charges likewise;
* the torch binding on CUDA tensors returns the C ABI's gradients;
* non-finite device input is rejected with AG_ERR_INVALID.
"""
import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu

K = 3


def _case(tmp_path, name="plain"):
    kw = {"plain": dict(n_atoms=500, npts=(16, 16, 16), seed=3, radius=12.0),
          "disorder": dict(n_atoms=400, npts=(14, 12, 16), seed=8, radius=11.0, pre_lines=["disorder_h"])}[name]
    kw = dict(kw)
    return make_case(tmp_path, name, kw.pop("n_atoms"), kw.pop("npts"), seed=kw.pop("seed"), radius=kw.pop("radius"),
                     **kw)


def _conformers(prob, seed=1):
    rng = np.random.default_rng(seed)
    c0 = prob.arrays["coord"].reshape(-1, 3)
    q0 = prob.arrays["charge"]
    coords = np.stack([c0 + (rng.normal(scale=0.3, size=c0.shape) if k else 0.0) for k in range(K)])
    charges = np.stack([q0 * (1.0 + 0.05 * k) for k in range(K)])
    return coords, charges


def _host_diff(ctx, job, prob, coords, charges, precision):
    from autogrid_b200 import Diff
    d = Diff(ctx, prob, precision, conformers=K)
    for k in range(K):
        rv, rv2 = job.bond_vectors(coords[k])
        d.set_atoms(coords[k], charges[k], rv, rv2, conformer=k)
    return d


def _device_diff(ctx, job, prob, coords, charges, precision):
    import torch
    from autogrid_b200 import Diff
    d = Diff(ctx, prob, precision, conformers=K)
    d.set_bonds(job)
    tc = torch.tensor(coords, dtype=torch.float64, device="cuda").contiguous()
    tq = torch.tensor(charges, dtype=torch.float64, device="cuda").contiguous()
    torch.cuda.synchronize()
    d.set_atoms_device(tc.data_ptr(), tq.data_ptr())
    return d


@pytest.mark.parametrize("name", ["plain", "disorder"])
def test_device_atoms_match_host_path(tmp_path, gpu_ctx, name):
    job, prob = _case(tmp_path, name)
    coords, charges = _conformers(prob)
    h = _host_diff(gpu_ctx, job, prob, coords, charges, "fp64")
    d = _device_diff(gpu_ctx, job, prob, coords, charges, "fp64")
    h.forward(); d.forward()
    assert np.array_equal(h.closest_h(), d.closest_h())
    mh, md = h.maps(), d.maps()
    scale = np.abs(mh).max()
    assert np.abs(mh - md).max() <= 1e-10 * scale, np.abs(mh - md).max() / scale
    # FP32 kernels on the same device state agree with their host-path twin too
    h32 = _host_diff(gpu_ctx, job, prob, coords, charges, "fp32")
    d32 = _device_diff(gpu_ctx, job, prob, coords, charges, "fp32")
    h32.forward(); d32.forward()
    m1, m2 = h32.maps().astype(np.float64), d32.maps().astype(np.float64)
    assert np.all(np.abs(m1 - m2) <= 1e-5 * np.maximum(1.0, np.abs(m1)))
    for x in (h, d, h32, d32):
        x.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_backward_device_matches_host_chain(tmp_path, gpu_ctx, precision):
    import torch
    job, prob = _case(tmp_path, "plain")
    coords, charges = _conformers(prob, seed=2)
    h = _host_diff(gpu_ctx, job, prob, coords, charges, precision)
    d = _device_diff(gpu_ctx, job, prob, coords, charges, precision)
    h.forward(); d.forward()
    rng = np.random.default_rng(4)
    w = rng.normal(size=h.shape).astype(h.dtype)
    g = h.backward(w)
    ref_c = np.stack([g["coord"][k] + job.bond_vectors_backward(coords[k], g["rvector"][k], g["rvector2"][k])
                      for k in range(K)])
    tw = torch.tensor(w, device="cuda").contiguous()
    gc = torch.empty((K, prob.n_atoms, 3), dtype=torch.float64, device="cuda")
    gq = torch.empty((K, prob.n_atoms), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    d.backward_device(tw.data_ptr(), gc.data_ptr(), gq.data_ptr())
    gc, gq = gc.cpu().numpy(), gq.cpu().numpy()
    tol = 1e-9 if precision == "fp64" else 1e-5
    assert np.linalg.norm(gc - ref_c) <= tol * np.linalg.norm(ref_c)
    assert np.linalg.norm(gq - g["charge"]) <= tol * np.linalg.norm(g["charge"])
    h.close(); d.close()


def test_torch_binding_on_cuda_tensors(tmp_path, gpu_ctx):
    import torch
    from autogrid_b200 import Diff, gradcheck
    from autogrid_b200.torch_maps import GridMaps
    job, prob = _case(tmp_path, "plain")
    fn = GridMaps(job, device=0, precision="fp64")
    c0 = prob.arrays["coord"].reshape(-1, 3) + np.random.default_rng(6).normal(scale=0.2, size=(prob.n_atoms, 3))
    coords = torch.tensor(c0, dtype=torch.float64, device="cuda", requires_grad=True)
    charges = torch.tensor(prob.arrays["charge"], dtype=torch.float64, device="cuda", requires_grad=True)
    maps = fn(coords, charges)
    w = torch.randn(prob.map_shape, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    (w * maps).sum().backward()
    assert coords.grad.is_cuda and charges.grad.is_cuda
    d = Diff(gpu_ctx, prob, "fp64")
    rv, rv2 = job.bond_vectors(c0)
    d.set_atoms(c0, prob.arrays["charge"], rv, rv2)
    d.forward()
    m = d.maps()
    np.testing.assert_allclose(maps.detach().cpu().numpy(), m, rtol=1e-10, atol=1e-10 * np.abs(m).max())
    gc, gq = gradcheck.full_gradient(job, d, c0, w.cpu().numpy())
    np.testing.assert_allclose(coords.grad.cpu().numpy(), gc, rtol=1e-8, atol=1e-9 * np.abs(gc).max())
    np.testing.assert_allclose(charges.grad.cpu().numpy(), gq, rtol=1e-8, atol=1e-9 * np.abs(gq).max())
    d.close()


def test_device_input_rejects_non_finite(tmp_path, gpu_ctx):
    import torch
    from autogrid_b200 import AutoGridError, Diff
    job, prob = _case(tmp_path, "plain")
    d = Diff(gpu_ctx, prob, "fp32")
    c = torch.tensor(prob.arrays["coord"].reshape(-1, 3), dtype=torch.float64, device="cuda")
    c[7, 1] = float("nan")
    torch.cuda.synchronize()
    with pytest.raises(AutoGridError):
        d.set_atoms_device(c.data_ptr())
    d.close()
