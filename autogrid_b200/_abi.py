"""ctypes mirror of include/autogrid_b200.h (the C ABI).

Structure layouts and function signatures here must match the header; the
test-suite checks that every function the header declares is exported by the
library and bound here.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_build" / "libautogrid_b200.so"

AG_A_DIV = 128
AG_NEINT = 1024
AG_NDIEL = 8192
AG_MAX_MAPS = 128
AG_MAX_REC_TYPES = 20
AG_MAX_ATOMS = 100000
AG_MAX_GRID_PTS = 1025

AG_OK = 0
STATUS_NAMES = {
    0: "AG_OK", 1: "AG_ERR_INVALID", 2: "AG_ERR_FATAL_INPUT", 3: "AG_ERR_NO_CLOSEST_H",
    4: "AG_ERR_UNSUPPORTED", 5: "AG_ERR_CUDA", 6: "AG_ERR_NO_DEVICE", 7: "AG_ERR_TOO_LARGE",
    8: "AG_ERR_IO", 9: "AG_ERR_TIMEOUT",
}
AG_PREC_FP32 = 0
AG_PREC_FP64 = 1
AG_TABLE_NEAREST = 0
AG_TABLE_LINEAR = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)
_u8p = C.POINTER(C.c_uint8)


class ag_problem(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32),
        ("coord", _dp), ("charge", _dp), ("vol", _dp), ("solpar", _dp),
        ("rec_type", _ip), ("hbond", _ip), ("rexp", _ip),
        ("rvector", _dp), ("rvector2", _dp), ("disorder", _u8p),
        ("n1", C.c_int32 * 3), ("ne", C.c_int32 * 3), ("spacing", C.c_double),
        ("n_rec_types", C.c_int32), ("n_atom_maps", C.c_int32), ("n_maps", C.c_int32),
        ("elec_map", C.c_int32), ("dsolv_map", C.c_int32),
        ("map_is_covalent", _ip), ("map_is_hbonder", _ip), ("map_hbond", _ip),
        ("map_solpar_probe", _dp), ("map_vol_probe", _dp),
        ("e_vdw_hb", _fp), ("sol_fn", _dp), ("r_epsilon_fn", _dp),
        ("dddiel", C.c_int32), ("invdielcal", C.c_double), ("coeff_estat", C.c_double),
        ("solpar_q", C.c_double), ("disorder_h", C.c_int32), ("hydrogen_type", C.c_int32),
        ("separate_desolvation_maps", C.c_int32),
        ("cov_pos", C.c_double * 3), ("cov_half_width", C.c_double), ("cov_barrier", C.c_double),
        ("floating_grid", C.c_int32), ("constriction_grid", C.c_int32),
        ("constriction_cutoff", C.c_double), ("report_collisions", C.c_int32),
    ]


class ag_opts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("table_mode", C.c_int32), ("autotune", C.c_int32),
                ("serial", C.c_int32), ("reserved", C.c_int32 * 4)]


class ag_stats(C.Structure):
    _fields_ = [("near_pairs", C.c_int64), ("fp64_fallbacks", C.c_int64), ("far_pairs", C.c_int64),
                ("gpu_launches", C.c_int32), ("reserved", C.c_int32), ("kernel_ms", C.c_double),
                ("far_ms", C.c_double), ("text_ms", C.c_double), ("text_bytes", C.c_int64),
                ("table_ms", C.c_double), ("far_edge_pairs", C.c_int64), ("far_fp32_bin_errors", C.c_int64),
                ("far_fp64_ties", C.c_int64), ("fixup_ms", C.c_double), ("near_ms", C.c_double)]


class ag_table_params(C.Structure):
    _fields_ = [("n_rec_types", C.c_int32), ("n_atom_maps", C.c_int32),
                ("cA", C.POINTER(C.c_double)), ("cB", C.POINTER(C.c_double)),
                ("Rij", C.POINTER(C.c_double)), ("epsij", C.POINTER(C.c_double)),
                ("xA", C.POINTER(C.c_int32)), ("xB", C.POINTER(C.c_int32)),
                ("map_is_covalent", C.POINTER(C.c_int32)),
                ("r_smooth", C.c_double), ("coeff_desolv", C.c_double), ("dddiel", C.c_int32)]


class ag_tuning(C.Structure):
    _fields_ = [("far_tile", C.c_int32), ("far_chunked", C.c_int32), ("near_shape", C.c_int32),
                ("candidates", C.c_int32), ("far_ms", C.c_double), ("near_ms", C.c_double),
                ("far_ms_default", C.c_double), ("near_ms_default", C.c_double)]


# name -> (restype, argtypes); every entry point declared in include/autogrid_b200.h
SIGNATURES = {
    "ag_last_error": (C.c_char_p, []),
    "ag_abi_version": (C.c_int32, []),
    "ag_context_create": (C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    "ag_context_destroy": (C.c_int, [C.c_void_p]),
    "ag_context_stats": (C.c_int, [C.c_void_p, C.POINTER(ag_stats)]),
    "ag_context_cached_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "ag_context_trim": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "ag_maps_compute": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts), C.c_void_p]),
    "ag_maps_compute_f64": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts), C.c_void_p]),
    "ag_plan_create": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts), C.POINTER(C.c_void_p)]),
    "ag_plan_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_plan_run_zslab": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "ag_maps_compute_zslab": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts), C.c_int32, C.c_int32,
                                        C.c_void_p]),
    "ag_plan_device_maps": (C.c_void_p, [C.c_void_p]),
    "ag_plan_points": (C.c_size_t, [C.c_void_p]),
    "ag_plan_download": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_plan_destroy": (C.c_int, [C.c_void_p]),
    "ag_tables_build": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_maps_format": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.c_void_p, C.c_int32,
                                 C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_maps_compute_text": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts),
                                       C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_batch_create": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(ag_problem)), C.c_int32, C.POINTER(ag_opts),
                                  C.POINTER(C.c_void_p)]),
    "ag_batch_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_batch_device_maps": (C.c_void_p, [C.c_void_p, C.c_int32]),
    "ag_batch_download": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "ag_batch_tuning": (C.c_int, [C.c_void_p, C.POINTER(ag_tuning)]),
    "ag_batch_destroy": (C.c_int, [C.c_void_p]),
    "ag_maps_compute_batch": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(ag_problem)), C.c_int32,
                                        C.POINTER(ag_opts), C.POINTER(C.c_void_p)]),
    "ag_job_load": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "ag_job_problem": (C.POINTER(ag_problem), [C.c_void_p]),
    "ag_job_write_maps_f32": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_job_write_maps_f64": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_job_write_text": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_job_fail": (None, [C.c_void_p, C.c_char_p]),
    "ag_job_free": (None, [C.c_void_p]),
    "ag_job_vina_problem": (C.c_int32, [C.c_void_p, C.POINTER(C.POINTER(ag_problem))]),
    "ag_job_bond_vectors": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_job_table_params": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "ag_job_bond_topology": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "ag_job_bond_vectors_backward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_diff_create": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts), C.POINTER(C.c_void_p)]),
    "ag_diff_create_batch": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.POINTER(ag_opts), C.c_int32,
                                       C.POINTER(C.c_void_p)]),
    "ag_diff_conformers": (C.c_int32, [C.c_void_p]),
    "ag_diff_set_atoms": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_diff_set_conformer": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_diff_forward": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p]),
    "ag_diff_device_maps": (C.c_void_p, [C.c_void_p]),
    "ag_diff_download": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_diff_closest_h": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_diff_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "ag_diff_set_bonds": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ag_diff_set_atoms_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_diff_backward_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ag_diff_timing": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "ag_diff_destroy": (C.c_int, [C.c_void_p]),
    "ag_emap_compute_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.POINTER(C.c_int32),
                                          C.c_double, C.c_int32, C.c_void_p, C.c_double, C.c_double,
                                          C.c_void_p, C.c_void_p]),
    # measurement and test helpers (include/autogrid_b200_diag.h)
    "ag_diag_peak_rates": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]),
    "ag_diag_rsqrt_error": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "ag_diag_far_bins": (C.c_int, [C.c_void_p, C.POINTER(ag_problem), C.c_int32, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
}

_lib = None


def load_library(path: Path | None = None) -> C.CDLL:
    """Load the native library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"autogrid_b200 native library missing at {p}; build it with `python -m autogrid_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class AutoGridError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def check(status: int) -> None:
    if status != AG_OK:
        msg = load_library().ag_last_error()
        raise AutoGridError(status, msg.decode() if msg else "")
