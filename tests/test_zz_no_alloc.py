"""The no-allocation electrostatic-map entry point (ag_emap_compute_noalloc).

It serves callers that may not allocate device memory (their process owns the
device through its own pool, or allocation is forbidden between requests); it
works only on caller-owned device buffers plus a fixed 32 MiB static scratch
array.  Checked against the regular entry point's e map (ag_maps_compute),
within the parity tolerance, on two calls in a row.  Collected last on
purpose: a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import make_case, tolerance_ok
from test_oracle_pinning import GOLDEN, load_golden

pytestmark = pytest.mark.gpu


def _bind(lib):
    fn = lib.ag_emap_compute_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_double, C.c_int32,
                   C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    return fn


def _problem(case, tmp_path):
    if case == "synthetic_10000":
        # 10,000 atoms on 41^3 points: many 512-atom chunks of the scratch's
        # partial sums, and a dense interior for the FP64 near-pair branch
        return make_case(tmp_path, "big", 10000, (40, 40, 40), seed=5)[1]
    path = [p for p in GOLDEN if p.stem == case][0]
    return load_golden(path, tmp_path)[2]


@pytest.mark.parametrize("case", ["basic_400", "types14_600", "constdiel_nbp", "synthetic_10000"])
def test_noalloc_emap_matches_regular_entry_point(case, tmp_path, built):
    import torch
    from autogrid_b200 import Context, load_library
    from autogrid_b200._abi import check
    prob = _problem(case, tmp_path)
    ctx = Context(0)
    regular = ctx.compute(prob, "fp32").reshape(prob.n_maps, -1)[prob.scalars["elec_map"]]
    ctx.close()
    fn = _bind(load_library())
    dev = torch.device("cuda:0")
    coord = torch.from_numpy(np.ascontiguousarray(prob.arrays["coord"])).to(dev)
    charge = torch.from_numpy(np.ascontiguousarray(prob.arrays["charge"])).to(dev)
    reps = torch.from_numpy(np.ascontiguousarray(prob.arrays["r_epsilon_fn"])).to(dev)
    out = torch.empty(prob.points, dtype=torch.float32, device=dev)
    n1 = (C.c_int32 * 3)(*prob.n1)
    sc = prob.scalars
    outs = []
    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(0)[0]
        check(fn(0, prob.n_atoms, coord.data_ptr(), charge.data_ptr(), n1, sc["spacing"], sc["dddiel"],
                 reps.data_ptr(), sc["invdielcal"], sc["coeff_estat"], out.data_ptr(), None))
        torch.cuda.synchronize()
        assert torch.cuda.current_device() == 0  # the caller's current device is left as it was
        if call == 1:  # the first call on a device resolves the static array's address
            assert torch.cuda.mem_get_info(0)[0] == free_before, "the no-alloc entry point changed free memory"
        got = out.cpu().numpy().astype(np.float64)
        assert np.isfinite(got).all()
        ok = tolerance_ok(got, regular.astype(np.float64))
        assert ok.all(), f"call {call}: {int((~ok).sum())} points outside tolerance"
        outs.append(got)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_oversized_grid(built):
    from autogrid_b200 import load_library
    fn = _bind(load_library())
    n1 = (C.c_int32 * 3)(1025, 1025, 1025)
    rc = fn(0, 10, None, None, n1, 0.375, 0, None, 4.0, 0.1406, C.c_void_p(16), None)
    assert rc == 1 or rc == 7  # AG_ERR_INVALID (null inputs) or AG_ERR_TOO_LARGE
    rc = fn(0, 0, None, None, n1, 0.375, 0, None, 4.0, 0.1406, C.c_void_p(16), None)
    assert rc == 7
    assert b"32 MiB" in load_library().ag_last_error()
