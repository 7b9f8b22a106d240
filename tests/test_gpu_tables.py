"""Energy tables built on the device (ag_tables_build) against the front
end's host tables (main.cpp:2040-2276, distdepdiel.cpp:30-57), and problems
whose tables live in device memory through every compute path.

* e_vdW_Hb: float-equal to the host's except where CUDA's pow rounds the last
  double bit differently and the float rounding follows it (counted; at most
  1 float ulp apart); sol_fn within 2 double ulps, r_epsilon_fn within 4e-15
  relative;
* maps from device-resident tables (one-shot, plan, FP64 twin, differentiable
  mode) equal the maps from the host tables to the parity bar;
* a zero exponent is the reference's fatal error (AG_ERR_FATAL_INPUT).
"""
import ctypes as C

import numpy as np
import pytest

from conftest import make_case, tolerance_ok
from test_oracle_pinning import GOLDEN, load_golden

pytestmark = pytest.mark.gpu
NEINT, NDIEL = 1024, 8192


def _device_tables(ctx, job, prob):
    import torch
    tp = job.table_params()
    n = max(1, prob.scalars["n_rec_types"] * prob.scalars["n_atom_maps"]) * NEINT
    e = torch.zeros(n, dtype=torch.float32, device="cuda")
    s = torch.zeros(NDIEL, dtype=torch.float64, device="cuda")
    r = torch.zeros(NDIEL, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ms = ctx.build_tables(tp, e.data_ptr(), s.data_ptr(), r.data_ptr() if prob.scalars["dddiel"] else None)
    return e, s, r, ms


def _ulps32(a, b):
    ia = a.astype(np.float32).view(np.int32).astype(np.int64)
    ib = b.astype(np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


CASES = [p for p in GOLDEN if p.stem in ("basic_400", "constdiel_nbp", "disorder_sep_cov", "types14_600",
                                          "noelec_odd")]


@pytest.mark.parametrize("path", CASES, ids=[p.stem for p in CASES])
def test_device_tables_match_host(path, tmp_path, gpu_ctx):
    _, job, prob = load_golden(path, tmp_path)
    e, s, r, ms = _device_tables(gpu_ctx, job, prob)
    n = prob.scalars["n_rec_types"] * prob.scalars["n_atom_maps"] * NEINT
    host_e = prob.arrays["e_vdw_hb"][:n]
    dev_e = e.cpu().numpy()[:n]
    u = _ulps32(dev_e, host_e)
    exact = float((u == 0).mean()) if n else 1.0
    print(f"{path.stem}: {exact:.6f} of {n} e_vdW_Hb entries float-equal, max {u.max() if n else 0} ulp; {ms:.3f} ms")
    assert exact >= 0.999 and (u.max() if n else 0) <= 1
    hs = prob.arrays["sol_fn"][:NDIEL]
    np.testing.assert_allclose(s.cpu().numpy(), hs, rtol=5e-16, atol=0)
    if prob.scalars["dddiel"]:
        # a 1-ulp difference of exp() grows through the cancellation in
        # A + B/(1 + k e^(-lambda B r)) (A < 0): a few ulps of 332/eps
        np.testing.assert_allclose(r.cpu().numpy(), prob.arrays["r_epsilon_fn"][:NDIEL], rtol=4e-15, atol=0)
    job.close()


@pytest.mark.parametrize("path", [p for p in GOLDEN if p.stem in ("disorder_sep_cov", "types14_600", "distance_maps",
                                                                   "constdiel_nbp")],
                         ids=lambda p: p.stem)
def test_maps_from_device_tables(path, tmp_path, gpu_ctx):
    from autogrid_b200 import Diff
    _, job, prob = load_golden(path, tmp_path)
    ref32 = gpu_ctx.compute(prob, "fp32").reshape(prob.n_out, -1).astype(np.float64)
    ref64 = gpu_ctx.compute(prob, "fp64").reshape(prob.n_out, -1)
    e, s, r, _ = _device_tables(gpu_ctx, job, prob)
    prob.device_tables = (e.data_ptr(), s.data_ptr(), r.data_ptr() if prob.scalars["dddiel"] else 0)
    got32 = gpu_ctx.compute(prob, "fp32").reshape(prob.n_out, -1).astype(np.float64)
    assert tolerance_ok(got32, ref32).all()
    print(f"{path.stem}: {float((got32 == ref32).mean()):.6f} of FP32 values identical")
    got64 = gpu_ctx.compute(prob, "fp64").reshape(prob.n_out, -1)
    assert np.all(np.abs(got64 - ref64) <= 1e-6 * np.maximum(1.0, np.abs(ref64)))
    plan = gpu_ctx.plan(prob)
    plan.run()
    np.testing.assert_array_equal(plan.download().reshape(prob.n_out, -1).astype(np.float64), got32)
    plan.close()
    if not (prob.scalars["floating_grid"] or prob.scalars["constriction_grid"]):
        d = Diff(gpu_ctx, prob, "fp64")
        d.forward()
        m_dev = d.maps()
        d.close()
        prob.device_tables = None
        h = Diff(gpu_ctx, prob, "fp64")
        h.forward()
        m_host = h.maps()
        h.close()
        assert np.all(np.abs(m_dev - m_host) <= 1e-6 * np.maximum(1.0, np.abs(m_host)))
    job.close()


def test_zero_exponent_is_fatal(tmp_path, gpu_ctx):
    import torch
    from autogrid_b200 import AutoGridError
    job, prob = make_case(tmp_path, "fatal", 200, (8, 8, 8), seed=2)
    tp = job.table_params()
    n = tp.n_rec_types * tp.n_atom_maps
    xA = np.ctypeslib.as_array(tp.xA, shape=(n,)).copy()
    xA[1] = 0
    tp.xA = xA.ctypes.data_as(C.POINTER(C.c_int32))
    e = torch.zeros(max(n, 1) * NEINT, dtype=torch.float32, device="cuda")
    s = torch.zeros(NDIEL, dtype=torch.float64, device="cuda")
    r = torch.zeros(NDIEL, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with pytest.raises(AutoGridError) as ei:
        gpu_ctx.build_tables(tp, e.data_ptr(), s.data_ptr(), r.data_ptr())
    assert ei.value.status == 2  # AG_ERR_FATAL_INPUT
    job.close()
