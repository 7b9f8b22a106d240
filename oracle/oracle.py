"""TEST INFRASTRUCTURE ONLY: Python binding of the FP64 C oracle and of the
reference binaries built under oracle/_ref/.  Only tests/, the smoke check and
bench.py's CPU-baseline / reference legs may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle_ag4.so"
REF_BIN = HERE / "_ref" / "autogrid4"
REF_FULLPREC_BIN = HERE / "_ref" / "autogrid4_fullprec"
# the same with the reference's USE_BHTREE switch (accepts 'map_receptor_interior off')
REF_BHTREE_BIN = HERE / "_ref" / "autogrid4_bhtree_fullprec"
# The reference source tree: AG_REFERENCE_SRC, or where this build's image
# mounts it.  Only the oracle build and the tests that read the reference's
# own test inputs use it; when it is absent those tests skip and the prebuilt
# oracle/_ref binaries (if any) are used as they are.
REFERENCE_SRC = Path(os.environ.get("AG_REFERENCE_SRC", "/root/reference"))

EDGE_BIN, EDGE_CUTOFF, EDGE_ANGLE, EDGE_CLOSEH = 1, 2, 4, 8


def build(ref: bool = True) -> None:
    """Build the oracle library (always) and the reference binaries (when the
    reference sources are present)."""
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    if ref and REFERENCE_SRC.exists():
        subprocess.run(["make", "-C", str(HERE), "-s", "-j8", "ref", f"REF={REFERENCE_SRC}"], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            build(ref=False)
        from autogrid_b200._abi import ag_problem
        _lib = C.CDLL(str(ORACLE_LIB))
        _lib.ag_oracle_points.restype = C.c_int32
        _lib.ag_oracle_points.argtypes = [C.POINTER(ag_problem), C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.ag_oracle_distance_maps.restype = C.c_int32
        _lib.ag_oracle_distance_maps.argtypes = [C.POINTER(ag_problem), C.c_int64, C.c_void_p, C.c_void_p]
        _lib.ag_oracle_points_lin.restype = C.c_int32
        _lib.ag_oracle_points_lin.argtypes = [C.POINTER(ag_problem), C.c_int64, C.c_void_p, C.c_void_p,
                                              C.c_void_p]
    return _lib


def oracle_points(problem, points: np.ndarray | None = None):
    """FP64 reference energies at `points` (linear indices; None = all).
    Returns (maps[n_maps, n_pts], edge_flags[n_pts])."""
    s = problem.struct()
    if points is None:
        n = problem.points
        idx_ptr = None
    else:
        points = np.ascontiguousarray(points, dtype=np.int64)
        n = int(points.shape[0])
        idx_ptr = points.ctypes.data_as(C.c_void_p)
    out = np.zeros((problem.n_maps, n), dtype=np.float64)
    flags = np.zeros(n, dtype=np.uint8)
    rc = lib().ag_oracle_points(C.byref(s), n, idx_ptr, out.ctypes.data_as(C.c_void_p),
                                flags.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise RuntimeError(f"oracle returned status {rc}")
    return out, flags


def oracle_distance_maps(problem, points: np.ndarray | None = None) -> np.ndarray:
    """FP64 floating-grid and constriction maps ([n_dist, n_pts]) of LOOP 1."""
    s = problem.struct()
    if points is None:
        n = problem.points
        idx_ptr = None
    else:
        points = np.ascontiguousarray(points, dtype=np.int64)
        n = int(points.shape[0])
        idx_ptr = points.ctypes.data_as(C.c_void_p)
    k = problem.n_out - problem.n_maps
    out = np.zeros((k, n), dtype=np.float64)
    rc = lib().ag_oracle_distance_maps(C.byref(s), n, idx_ptr, out.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise RuntimeError(f"oracle returned status {rc}")
    return out


def oracle_points_lin(problem, points: np.ndarray | None = None, closest_h: np.ndarray | None = None):
    """FP64 energies of the differentiable (linear-table) mode at `points`
    (linear indices; None = all), with the closest DS/D1 atom of each point
    frozen to closest_h (per point; None = searched).  Returns maps[n_maps, n_pts]."""
    s = problem.struct()
    if points is None:
        n = problem.points
        idx_ptr = None
    else:
        points = np.ascontiguousarray(points, dtype=np.int64)
        n = int(points.shape[0])
        idx_ptr = points.ctypes.data_as(C.c_void_p)
    ch_ptr = None
    if closest_h is not None:
        closest_h = np.ascontiguousarray(closest_h, dtype=np.int32)
        assert closest_h.shape[0] == n
        ch_ptr = closest_h.ctypes.data_as(C.c_void_p)
    out = np.zeros((problem.n_maps, n), dtype=np.float64)
    rc = lib().ag_oracle_points_lin(C.byref(s), n, idx_ptr, ch_ptr, out.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise RuntimeError(f"oracle returned status {rc}")
    return out


def read_map(path: str | Path) -> np.ndarray:
    """Values of an AutoGrid .map file (6 header lines skipped)."""
    with open(path) as f:
        lines = f.read().split("\n")
    return np.array([float(v) for v in lines[6:] if v.strip()], dtype=np.float64)
