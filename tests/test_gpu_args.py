"""Entry points that hand a caller's pointer to a kernel reject host memory
with AG_ERR_INVALID before any launch (cudaPointerGetAttributes), so a wrong
pointer is an argument error and never reaches the GPU."""
import ctypes as C

import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu
AG_ERR_INVALID = 1


def test_format_rejects_host_maps(tmp_path, gpu_ctx):
    from autogrid_b200 import AutoGridError
    _, prob = make_case(tmp_path, "a", 200, (8, 8, 8), seed=1)
    host = np.zeros(prob.n_out * prob.points, dtype=np.float32)
    with pytest.raises(AutoGridError) as ei:
        gpu_ctx.format(prob, host.ctypes.data, 4)
    assert ei.value.status == AG_ERR_INVALID


def test_diff_device_calls_reject_host_pointers(tmp_path, gpu_ctx):
    import torch
    from autogrid_b200 import AutoGridError, Diff
    _, prob = make_case(tmp_path, "b", 200, (8, 8, 8), seed=2)
    d = Diff(gpu_ctx, prob, "fp32")
    coord = np.ascontiguousarray(prob.arrays["coord"], dtype=np.float64)
    with pytest.raises(AutoGridError) as ei:
        d.set_atoms_device(coord.ctypes.data)
    assert ei.value.status == AG_ERR_INVALID
    out = np.zeros(prob.n_maps * prob.points, dtype=np.float32)
    with pytest.raises(AutoGridError) as ei:
        d.forward(device_out=out.ctypes.data)
    assert ei.value.status == AG_ERR_INVALID
    d.forward()
    g = torch.zeros(prob.map_shape, dtype=torch.float32, device="cuda")
    gc = np.zeros((prob.n_atoms, 3))
    torch.cuda.synchronize()
    with pytest.raises(AutoGridError) as ei:
        d.backward_device(g.data_ptr(), gc.ctypes.data, None)
    assert ei.value.status == AG_ERR_INVALID
    d.close()


def test_noalloc_rejects_host_buffers(built):
    from autogrid_b200 import load_library
    fn = load_library().ag_emap_compute_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_double, C.c_int32,
                   C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    coord = np.zeros(30); charge = np.zeros(10); emap = np.zeros(27, dtype=np.float32)
    n1 = (C.c_int32 * 3)(3, 3, 3)
    st = fn(0, 10, coord.ctypes.data, charge.ctypes.data, n1, 0.375, 0, None, 332.0 / 40.0, 0.1465,
            emap.ctypes.data, None)
    assert st == AG_ERR_INVALID
