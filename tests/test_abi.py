"""The C ABI library: loads without a GPU, exports every declared entry point,
and reports the absence of a device as a status code."""
import ctypes as C
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(ag_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("ag_maps_compute", "ag_maps_compute_f64", "ag_plan_create", "ag_job_load", "ag_context_create"):
        assert n in names


def test_library_exports_every_declared_symbol(built):
    from autogrid_b200._abi import LIB_PATH, SIGNATURES
    lib = C.CDLL(str(LIB_PATH))
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
        assert name in SIGNATURES, f"{name} not bound in autogrid_b200/_abi.py"


def test_abi_version(built):
    from autogrid_b200 import load_library
    assert load_library().ag_abi_version() == 2


def test_context_without_device_is_a_status(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from autogrid_b200 import AutoGridError, Context
    with pytest.raises(AutoGridError) as e:
        Context(0)
    assert e.value.status == 6  # AG_ERR_NO_DEVICE
