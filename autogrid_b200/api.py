"""Python host API over the C ABI.

Mirrors the reference's one operation -- `autogrid4 -p x.gpf -l x.glg`
(main.cpp:214-3582) -- as `run_gpf()`, and exposes its hot path
(main.cpp:2805-3464) as `Context.compute()` on a `Problem`.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import AutoGridError, ag_opts, ag_problem, ag_stats, check, load_library

_PREC = {"fp32": _abi.AG_PREC_FP32, "fp64": _abi.AG_PREC_FP64}


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


class Problem:
    """Owner of the numpy arrays behind one ag_problem.

    Build it from a loaded GPF job (`Job.problem()`), or from arrays.  Array
    names and meaning follow include/autogrid_b200.h.
    """

    ARRAYS = {
        "coord": np.float64, "charge": np.float64, "vol": np.float64, "solpar": np.float64,
        "rec_type": np.int32, "hbond": np.int32, "rexp": np.int32, "rvector": np.float64,
        "rvector2": np.float64, "disorder": np.uint8, "map_is_covalent": np.int32,
        "map_is_hbonder": np.int32, "map_hbond": np.int32, "map_solpar_probe": np.float64,
        "map_vol_probe": np.float64, "e_vdw_hb": np.float32, "sol_fn": np.float64,
        "r_epsilon_fn": np.float64,
    }
    SCALARS = ("n_rec_types", "n_atom_maps", "n_maps", "elec_map", "dsolv_map", "spacing", "dddiel",
               "invdielcal", "coeff_estat", "solpar_q", "disorder_h", "hydrogen_type",
               "separate_desolvation_maps", "cov_half_width", "cov_barrier", "floating_grid",
               "constriction_grid", "constriction_cutoff", "report_collisions")

    def __init__(self, **kw):
        self.arrays = {}
        for name, dt in self.ARRAYS.items():
            v = kw.get(name)
            self.arrays[name] = None if v is None else np.ascontiguousarray(np.asarray(v, dtype=dt))
        self.n1 = tuple(int(v) for v in kw["n1"])
        self.ne = tuple(int(v) for v in kw.get("ne", [(n - 1) // 2 for n in self.n1]))
        self.scalars = {k: kw[k] for k in self.SCALARS if k in kw}
        self.cov_pos = tuple(float(v) for v in kw.get("cov_pos", (0.0, 0.0, 0.0)))
        self.n_atoms = 0 if self.arrays["charge"] is None else int(self.arrays["charge"].shape[0])
        self._struct = None

    @property
    def n_maps(self) -> int:
        return int(self.scalars["n_maps"])

    @property
    def points(self) -> int:
        return self.n1[0] * self.n1[1] * self.n1[2]

    @property
    def n_out(self) -> int:
        """Output arrays: the n_maps energy maps, then the floating-grid and
        constriction maps when requested."""
        return (self.n_maps + int(bool(self.scalars.get("floating_grid", 0)))
                + int(bool(self.scalars.get("constriction_grid", 0))))

    @property
    def map_shape(self) -> tuple:
        return (self.n_out, self.n1[2], self.n1[1], self.n1[0])

    def struct(self) -> ag_problem:
        a = self.arrays
        s = ag_problem()
        s.n_atoms = self.n_atoms
        s.coord = _ptr(a["coord"], C.c_double)
        s.charge = _ptr(a["charge"], C.c_double)
        s.vol = _ptr(a["vol"], C.c_double)
        s.solpar = _ptr(a["solpar"], C.c_double)
        s.rec_type = _ptr(a["rec_type"], C.c_int32)
        s.hbond = _ptr(a["hbond"], C.c_int32)
        s.rexp = _ptr(a["rexp"], C.c_int32)
        s.rvector = _ptr(a["rvector"], C.c_double)
        s.rvector2 = _ptr(a["rvector2"], C.c_double)
        s.disorder = _ptr(a["disorder"], C.c_uint8)
        for i in range(3):
            s.n1[i] = self.n1[i]
            s.ne[i] = self.ne[i]
            s.cov_pos[i] = self.cov_pos[i]
        s.map_is_covalent = _ptr(a["map_is_covalent"], C.c_int32)
        s.map_is_hbonder = _ptr(a["map_is_hbonder"], C.c_int32)
        s.map_hbond = _ptr(a["map_hbond"], C.c_int32)
        s.map_solpar_probe = _ptr(a["map_solpar_probe"], C.c_double)
        s.map_vol_probe = _ptr(a["map_vol_probe"], C.c_double)
        s.e_vdw_hb = _ptr(a["e_vdw_hb"], C.c_float)
        s.sol_fn = _ptr(a["sol_fn"], C.c_double)
        s.r_epsilon_fn = _ptr(a["r_epsilon_fn"], C.c_double)
        dt = getattr(self, "device_tables", None)
        if dt is not None:  # (e_vdw_hb, sol_fn, r_epsilon_fn) device pointers, e.g. from ag_tables_build
            s.e_vdw_hb = C.cast(C.c_void_p(int(dt[0])), C.POINTER(C.c_float))
            s.sol_fn = C.cast(C.c_void_p(int(dt[1])), C.POINTER(C.c_double))
            s.r_epsilon_fn = C.cast(C.c_void_p(int(dt[2])), C.POINTER(C.c_double)) if dt[2] else None
        for k, v in self.scalars.items():
            setattr(s, k, v)
        self._struct = s  # arrays stay alive with self
        return s

    def bytes_h2d(self) -> int:
        return int(sum(v.nbytes for v in self.arrays.values() if v is not None))

    @classmethod
    def from_struct(cls, s: ag_problem) -> "Problem":
        """Copy a problem the front end built (ag_job_problem) into numpy arrays."""
        n = s.n_atoms
        nam = s.n_atom_maps
        nrt = max(s.n_rec_types, 1)

        def arr(ptr, count, dt):
            if count == 0 or not ptr:
                return np.zeros(count, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        kw = dict(
            coord=arr(s.coord, 3 * n, np.float64).reshape(n, 3), charge=arr(s.charge, n, np.float64),
            vol=arr(s.vol, n, np.float64), solpar=arr(s.solpar, n, np.float64),
            rec_type=arr(s.rec_type, n, np.int32), hbond=arr(s.hbond, n, np.int32),
            rexp=arr(s.rexp, n, np.int32), rvector=arr(s.rvector, 3 * n, np.float64).reshape(n, 3),
            rvector2=arr(s.rvector2, 3 * n, np.float64).reshape(n, 3),
            disorder=arr(s.disorder, n, np.uint8),
            map_is_covalent=arr(s.map_is_covalent, max(nam, 1), np.int32),
            map_is_hbonder=arr(s.map_is_hbonder, max(nam, 1), np.int32),
            map_hbond=arr(s.map_hbond, max(nam, 1), np.int32),
            map_solpar_probe=arr(s.map_solpar_probe, max(nam, 1), np.float64),
            map_vol_probe=arr(s.map_vol_probe, max(nam, 1), np.float64),
            e_vdw_hb=arr(s.e_vdw_hb, nrt * max(nam, 1) * _abi.AG_NEINT, np.float32),
            sol_fn=arr(s.sol_fn, _abi.AG_NDIEL, np.float64),
            r_epsilon_fn=arr(s.r_epsilon_fn, _abi.AG_NDIEL, np.float64),
            n1=list(s.n1), ne=list(s.ne), cov_pos=list(s.cov_pos),
        )
        for k in cls.SCALARS:
            kw[k] = getattr(s, k)
        return cls(**kw)


class Job:
    """A parsed GPF: front end of `autogrid4 -p gpf -l glg` (ag_job_load)."""

    def __init__(self, gpf: str, glg: str | None = None):
        lib = load_library()
        h = C.c_void_p()
        check(lib.ag_job_load(os.fsencode(gpf), os.fsencode(glg) if glg else None, C.byref(h)))
        self._h = h
        self._lib = lib
        self.n_atoms = int(lib.ag_job_problem(h).contents.n_atoms)

    def problem(self) -> Problem:
        return Problem.from_struct(self._lib.ag_job_problem(self._h).contents)

    def write_maps(self, maps: np.ndarray) -> None:
        m = np.ascontiguousarray(maps)
        if m.dtype == np.float64:
            check(self._lib.ag_job_write_maps_f64(self._h, m.ctypes.data_as(C.c_void_p)))
        else:
            m = np.ascontiguousarray(m, dtype=np.float32)
            check(self._lib.ag_job_write_maps_f32(self._h, m.ctypes.data_as(C.c_void_p)))

    def write_text(self, mt: "MapText") -> None:
        """Write the map files and GLG summary from device-formatted bodies
        (ag_job_write_text)."""
        b = np.ascontiguousarray(mt.map_bytes, dtype=np.uint64)
        lo = np.ascontiguousarray(mt.emin, dtype=np.float64)
        hi = np.ascontiguousarray(mt.emax, dtype=np.float64)
        check(self._lib.ag_job_write_text(self._h, C.c_void_p(mt.ptr), b.ctypes.data_as(C.c_void_p),
                                          lo.ctypes.data_as(C.c_void_p), hi.ctypes.data_as(C.c_void_p)))

    def vina_problem(self) -> Problem:
        """The job with Vina-potential tables (ag_job_vina_problem): atom maps
        only, plain sums, no desolvation."""
        out = C.POINTER(ag_problem)()
        check(self._lib.ag_job_vina_problem(self._h, C.byref(out)))
        return Problem.from_struct(out.contents)

    def bond_vectors(self, coord: np.ndarray | None = None) -> tuple:
        """(rvector, rvector2) [N,3] at coord [N,3] (centred frame), with the
        bonded neighbours found at load time (ag_job_bond_vectors)."""
        n = self.n_atoms
        rv = np.zeros((n, 3)); rv2 = np.zeros((n, 3))
        c = None if coord is None else np.ascontiguousarray(coord, dtype=np.float64).reshape(n, 3)
        check(self._lib.ag_job_bond_vectors(self._h, None if c is None else c.ctypes.data_as(C.c_void_p),
                                            rv.ctypes.data_as(C.c_void_p), rv2.ctypes.data_as(C.c_void_p)))
        return rv, rv2

    def bond_vectors_backward(self, coord, g_rvector, g_rvector2) -> np.ndarray:
        """d(rvector, rvector2)/d(coord)^T (g_rvector, g_rvector2), [N,3] FP64."""
        n = self.n_atoms
        c = np.ascontiguousarray(coord, dtype=np.float64).reshape(n, 3)
        g1 = np.ascontiguousarray(g_rvector, dtype=np.float64).reshape(n, 3)
        g2 = np.ascontiguousarray(g_rvector2, dtype=np.float64).reshape(n, 3)
        out = np.zeros((n, 3))
        check(self._lib.ag_job_bond_vectors_backward(self._h, c.ctypes.data_as(C.c_void_p),
                                                     g1.ctypes.data_as(C.c_void_p), g2.ctypes.data_as(C.c_void_p),
                                                     out.ctypes.data_as(C.c_void_p)))
        return out

    def table_params(self) -> "_abi.ag_table_params":
        """The job's table parameters for ag_tables_build (ag_job_table_params;
        the arrays belong to the job)."""
        tp = _abi.ag_table_params()
        check(self._lib.ag_job_table_params(self._h, C.byref(tp)))
        return tp

    def bond_topology(self) -> np.ndarray:
        """int32 [N, 7]: kind (AG_BOND_*), i1, i2, nb, nbr[3] per atom."""
        out = np.zeros((self.n_atoms, 7), dtype=np.int32)
        check(self._lib.ag_job_bond_topology(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def fail(self, message: str) -> None:
        self._lib.ag_job_fail(self._h, message.encode())

    def close(self) -> None:
        if self._h:
            self._lib.ag_job_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class MapText:
    """Map-file bodies formatted on the device (ag_maps_format).  `ptr` is the
    context's pinned host buffer: valid until the context's next text call."""
    ptr: int
    map_bytes: np.ndarray  # uint64, one entry per output map
    emin: np.ndarray       # extrema of each energy map
    emax: np.ndarray

    @property
    def total(self) -> int:
        return int(self.map_bytes.sum())

    def body(self, k: int) -> bytes:
        off = int(self.map_bytes[:k].sum())
        return C.string_at(self.ptr + off, int(self.map_bytes[k]))

    def tobytes(self) -> bytes:
        return C.string_at(self.ptr, self.total)


def _text_call(fn, problem: Problem, *head) -> MapText:
    s = problem.struct()
    ptr = C.c_void_p()
    nb = np.zeros(problem.n_out, dtype=np.uint64)
    lo = np.zeros(max(1, problem.n_maps)); hi = np.zeros(max(1, problem.n_maps))
    check(fn(head[0], C.byref(s), *head[1:], C.byref(ptr), nb.ctypes.data_as(C.c_void_p),
             lo.ctypes.data_as(C.c_void_p), hi.ctypes.data_as(C.c_void_p)))
    return MapText(int(ptr.value or 0), nb, lo[:problem.n_maps], hi[:problem.n_maps])


@dataclass
class Stats:
    near_pairs: int
    fp64_fallbacks: int
    far_pairs: int
    gpu_launches: int
    kernel_ms: float
    far_ms: float
    text_ms: float = 0.0
    text_bytes: int = 0
    far_edge_pairs: int = 0
    far_fp32_bin_errors: int = 0
    far_fp64_ties: int = 0
    fixup_ms: float = 0.0
    near_ms: float = 0.0


class Context:
    """A CUDA device context of the map engine (ag_context)."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        h = C.c_void_p()
        check(self._lib.ag_context_create(int(device), C.byref(h)))
        self._h = h

    def compute(self, problem: Problem, precision: str = "fp32", out: np.ndarray | None = None) -> np.ndarray:
        """Compute every map of `problem`; returns [n_maps, n1z, n1y, n1x]."""
        prec = _PREC[precision]
        dt = np.float64 if prec == _abi.AG_PREC_FP64 else np.float32
        if out is None:
            out = np.empty(problem.map_shape, dtype=dt)
        if out.dtype != dt or not out.flags.c_contiguous or out.size != int(np.prod(problem.map_shape)):
            raise ValueError("out must be a C-contiguous array of the map shape and precision")
        opts = ag_opts(precision=prec, table_mode=_abi.AG_TABLE_NEAREST)
        s = problem.struct()
        fn = self._lib.ag_maps_compute_f64 if prec == _abi.AG_PREC_FP64 else self._lib.ag_maps_compute
        check(fn(self._h, C.byref(s), C.byref(opts), out.ctypes.data_as(C.c_void_p)))
        return out

    def compute_zslab(self, problem: Problem, z0: int, z1: int, out: np.ndarray | None = None) -> np.ndarray:
        """FP32 maps of grid planes [z0, z1) (ag_maps_compute_zslab); returns
        [n_out, z1 - z0, n1y, n1x]."""
        shape = (problem.n_out, int(z1) - int(z0), problem.n1[1], problem.n1[0])
        if out is None:
            out = np.empty(shape, dtype=np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.shape != shape:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {shape}")
        opts = ag_opts(precision=_abi.AG_PREC_FP32, table_mode=_abi.AG_TABLE_NEAREST)
        s = problem.struct()
        check(self._lib.ag_maps_compute_zslab(self._h, C.byref(s), C.byref(opts), int(z0), int(z1),
                                              out.ctypes.data_as(C.c_void_p)))
        return out

    def compute_text(self, problem: Problem, precision: str = "fp32") -> MapText:
        """Compute the maps and format their map-file bodies on the device
        (ag_maps_compute_text)."""
        opts = ag_opts(precision=_PREC[precision], table_mode=_abi.AG_TABLE_NEAREST)
        return _text_call(self._lib.ag_maps_compute_text, problem, self._h, C.byref(opts))

    def build_tables(self, params, e_vdw_hb: int, sol_fn: int, r_epsilon_fn: int | None) -> float:
        """Energy tables on the device (ag_tables_build) into the given buffers
        (host or device addresses); returns the kernels' device time in ms."""
        check(self._lib.ag_tables_build(self._h, C.byref(params), C.c_void_p(int(e_vdw_hb)), C.c_void_p(int(sol_fn)),
                                        None if not r_epsilon_fn else C.c_void_p(int(r_epsilon_fn))))
        st = ag_stats()
        check(self._lib.ag_context_stats(self._h, C.byref(st)))
        return st.table_ms

    def format(self, problem: Problem, device_ptr: int, elem_size: int = 4) -> MapText:
        """Format device-resident maps of `problem`'s layout (ag_maps_format)."""
        return _text_call(self._lib.ag_maps_format, problem, self._h, C.c_void_p(int(device_ptr)),
                          C.c_int32(int(elem_size)))

    def stats(self) -> Stats:
        st = ag_stats()
        check(self._lib.ag_context_stats(self._h, C.byref(st)))
        return Stats(st.near_pairs, st.fp64_fallbacks, st.far_pairs, st.gpu_launches, st.kernel_ms, st.far_ms,
                     st.text_ms, st.text_bytes, st.far_edge_pairs, st.far_fp32_bin_errors, st.far_fp64_ties,
                     st.fixup_ms, st.near_ms)

    def cached_bytes(self) -> int:
        """Device memory the context keeps for later batches (ag_context_cached_bytes)."""
        v = C.c_int64()
        check(self._lib.ag_context_cached_bytes(self._h, C.byref(v)))
        return int(v.value)

    def trim(self) -> int:
        """Free the context's cached batch memory; returns the bytes freed (ag_context_trim)."""
        v = C.c_int64()
        check(self._lib.ag_context_trim(self._h, C.byref(v)))
        return int(v.value)

    def far_bins(self, problem: Problem, points) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Far-field table bins of the given grid points (linear indices, X
        fastest) against every atom, with the far kernel's arithmetic
        (ag_diag_far_bins): (bin_used, bin_fp32, flags), each [n_points, n_atoms].
        bin_used is -1 for pairs nearer than 8 A (the near-field kernel's)."""
        pts = np.ascontiguousarray(points, dtype=np.int64)
        shape = (pts.size, problem.n_atoms)
        used = np.empty(shape, np.int32)
        fp32 = np.empty(shape, np.int32)
        flags = np.empty(shape, np.int32)
        s = problem.struct()
        check(self._lib.ag_diag_far_bins(self._h, C.byref(s), int(pts.size), pts.ctypes.data_as(C.c_void_p),
                                         used.ctypes.data_as(C.c_void_p), fp32.ctypes.data_as(C.c_void_p),
                                         flags.ctypes.data_as(C.c_void_p)))
        return used, fp32, flags

    def plan(self, problem: Problem, serial: bool = False) -> "Plan":
        """Device-resident plan; serial=True runs every kernel in sequence on one
        stream (same work, for timing kernels alone)."""
        return Plan(self, problem, serial)

    def close(self) -> None:
        if self._h:
            self._lib.ag_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Diff:
    """Differentiable mode (ag_diff_*): maps with linearly interpolated tables
    and their hand-written adjoint.  Arrays are FP64 numpy in the problem's
    centred frame; maps and map gradients are in the chosen precision.  With
    conformers > 1 the object holds that many coordinate sets of the receptor,
    evaluated together; maps, closest-H indices and gradients gain a leading
    conformer axis."""

    def __init__(self, ctx: Context, problem: Problem, precision: str = "fp32", conformers: int = 1):
        self.ctx = ctx
        self.problem = problem
        self._lib = ctx._lib
        prec = _PREC[precision]
        self.dtype = np.float64 if prec == _abi.AG_PREC_FP64 else np.float32
        self.conformers = int(conformers)
        self.shape = problem.map_shape if self.conformers == 1 else (self.conformers,) + problem.map_shape
        self.n_atoms = problem.n_atoms
        opts = ag_opts(precision=prec, table_mode=_abi.AG_TABLE_LINEAR)
        s = problem.struct()
        h = C.c_void_p()
        check(self._lib.ag_diff_create_batch(ctx._h, C.byref(s), C.byref(opts), self.conformers, C.byref(h)))
        self._h = h

    @staticmethod
    def _ptr(a, n, cols=None):
        if a is None:
            return None, None
        shape = (n,) if cols is None else (n, cols)
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))
        return arr, arr.ctypes.data_as(C.c_void_p)

    def set_atoms(self, coord=None, charge=None, rvector=None, rvector2=None, conformer: int = 0) -> None:
        n = self.n_atoms
        c, pc = self._ptr(coord, n, 3)
        q, pq = self._ptr(charge, n)
        r1, p1 = self._ptr(rvector, n, 3)
        r2, p2 = self._ptr(rvector2, n, 3)
        check(self._lib.ag_diff_set_conformer(self._h, int(conformer), pc, pq, p1, p2))

    def forward(self, keep_closest_h: bool = False, device_out: int | None = None) -> None:
        """Compute the maps (into device_out, a device pointer, or the object's buffer)."""
        check(self._lib.ag_diff_forward(self._h, int(bool(keep_closest_h)),
                                        None if device_out is None else C.c_void_p(int(device_out))))

    def maps(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        check(self._lib.ag_diff_download(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def closest_h(self) -> np.ndarray:
        P = int(np.prod(self.problem.map_shape[1:]))
        out = np.empty(P * self.conformers, dtype=np.int32)
        check(self._lib.ag_diff_closest_h(self._h, out.ctypes.data_as(C.c_void_p)))
        return out if self.conformers == 1 else out.reshape(self.conformers, P)

    def backward(self, grad_maps=None, device_ptr: int | None = None) -> dict:
        """Adjoint of the last forward for dL/d(maps) given as a host array or a
        device pointer.  Returns FP64 dL/d(coord) (pair terms only), charge,
        rvector, rvector2."""
        n, k = self.n_atoms, self.conformers
        lead = () if k == 1 else (k,)
        gc = np.zeros(lead + (n, 3)); gq = np.zeros(lead + (n,))
        g1 = np.zeros(lead + (n, 3)); g2 = np.zeros(lead + (n, 3))
        if device_ptr is not None:
            src, on_dev = C.c_void_p(int(device_ptr)), 1
        else:
            g = np.ascontiguousarray(grad_maps, dtype=self.dtype)
            if g.size != int(np.prod(self.shape)):
                raise ValueError("grad_maps must have the map shape")
            src, on_dev = g.ctypes.data_as(C.c_void_p), 0
        check(self._lib.ag_diff_backward(self._h, src, on_dev, gc.ctypes.data_as(C.c_void_p),
                                         gq.ctypes.data_as(C.c_void_p), g1.ctypes.data_as(C.c_void_p),
                                         g2.ctypes.data_as(C.c_void_p)))
        return {"coord": gc, "charge": gq, "rvector": g1, "rvector2": g2}

    def set_bonds(self, job: "Job") -> None:
        """Attach the job's bond topology (ag_job_bond_topology) so that
        device-resident updates rebuild the bond vectors on the device."""
        topo = job.bond_topology()
        check(self._lib.ag_diff_set_bonds(self._h, topo.ctypes.data_as(C.c_void_p)))

    def set_atoms_device(self, coord_ptr: int, charge_ptr: int | None = None) -> None:
        """Every conformer's coordinates [K][N][3] (and charges [K][N]) from
        device pointers to FP64 arrays (ag_diff_set_atoms_device)."""
        check(self._lib.ag_diff_set_atoms_device(self._h, C.c_void_p(int(coord_ptr)),
                                                 None if charge_ptr is None else C.c_void_p(int(charge_ptr))))

    def backward_device(self, grad_ptr: int, g_coord_ptr: int | None, g_charge_ptr: int | None) -> None:
        """Adjoint with the map gradient and the FP64 outputs [K][N][3], [K][N]
        in device memory (ag_diff_backward_device)."""
        ptr = lambda v: None if v is None else C.c_void_p(int(v))  # noqa: E731
        check(self._lib.ag_diff_backward_device(self._h, C.c_void_p(int(grad_ptr)), ptr(g_coord_ptr),
                                                ptr(g_charge_ptr)))

    def timing(self) -> tuple:
        """(forward_ms, closest_h_ms, backward_ms) of the last calls (device events)."""
        f, c, b = C.c_float(), C.c_float(), C.c_float()
        check(self._lib.ag_diff_timing(self._h, C.byref(f), C.byref(c), C.byref(b)))
        return f.value, c.value, b.value

    def close(self) -> None:
        if self._h:
            self._lib.ag_diff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """Device-resident problem: upload once, run many times (ag_plan)."""

    def __init__(self, ctx: Context, problem: Problem, serial: bool = False):
        self.ctx = ctx
        self.problem = problem
        self._lib = ctx._lib
        h = C.c_void_p()
        opts = ag_opts(precision=_abi.AG_PREC_FP32, table_mode=_abi.AG_TABLE_NEAREST, serial=int(bool(serial)))
        s = problem.struct()
        check(self._lib.ag_plan_create(ctx._h, C.byref(s), C.byref(opts), C.byref(h)))
        self._h = h

    def run(self, stream: int | None = None) -> None:
        check(self._lib.ag_plan_run(self._h, C.c_void_p(stream) if stream else None))

    def run_zslab(self, z0: int, z1: int, stream: int | None = None) -> None:
        """Run grid planes [z0, z1) only (ag_plan_run_zslab)."""
        check(self._lib.ag_plan_run_zslab(self._h, int(z0), int(z1), C.c_void_p(stream) if stream else None))

    def device_maps_ptr(self) -> int:
        return int(self._lib.ag_plan_device_maps(self._h) or 0)

    def format(self) -> MapText:
        """Map-file bodies of the plan's device maps (ag_maps_format)."""
        return self.ctx.format(self.problem, self.device_maps_ptr(), 4)

    def download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.problem.map_shape, dtype=np.float32)
        check(self._lib.ag_plan_download(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def close(self) -> None:
        if self._h:
            self._lib.ag_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent problems computed by one persistent launch per kernel
    kind, graph-captured, and (by default) autotuned at creation (ag_batch)."""

    def __init__(self, ctx: Context, problems: list, autotune: bool = True):
        self.ctx = ctx
        self.problems = list(problems)
        self._lib = ctx._lib
        self._structs = [p.struct() for p in self.problems]
        arr = (C.POINTER(ag_problem) * len(self._structs))(*[C.pointer(s) for s in self._structs])
        opts = ag_opts(precision=_abi.AG_PREC_FP32, table_mode=_abi.AG_TABLE_NEAREST, autotune=int(autotune))
        h = C.c_void_p()
        check(self._lib.ag_batch_create(ctx._h, arr, len(self.problems), C.byref(opts), C.byref(h)))
        self._h = h

    def run(self, stream: int | None = None) -> None:
        check(self._lib.ag_batch_run(self._h, C.c_void_p(stream) if stream else None))

    def download(self, i: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.problems[i].map_shape, dtype=np.float32)
        check(self._lib.ag_batch_download(self._h, int(i), out.ctypes.data_as(C.c_void_p)))
        return out

    def tuning(self) -> dict:
        t = _abi.ag_tuning()
        check(self._lib.ag_batch_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def close(self) -> None:
        if self._h:
            self._lib.ag_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def compute_batch(ctx: Context, problems: list, outs: list | None = None) -> list:
    """One-shot batched computation (ag_maps_compute_batch): host inputs in,
    host maps out (into `outs` when given), no autotuning."""
    structs = [p.struct() for p in problems]
    arr = (C.POINTER(ag_problem) * len(structs))(*[C.pointer(s) for s in structs])
    if outs is None:
        outs = [np.empty(p.map_shape, dtype=np.float32) for p in problems]
    for p, o in zip(problems, outs):
        if o.dtype != np.float32 or not o.flags.c_contiguous or o.size != int(np.prod(p.map_shape)):
            raise ValueError("each output must be a C-contiguous float32 array of its problem's map shape")
    ptrs = (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
    opts = ag_opts(precision=_abi.AG_PREC_FP32, table_mode=_abi.AG_TABLE_NEAREST)
    check(ctx._lib.ag_maps_compute_batch(ctx._h, arr, len(problems), C.byref(opts), ptrs))
    return outs


def run_gpf(gpf: str, glg: str | None = None, precision: str = "fp32", device: int = 0) -> np.ndarray:
    """Drop-in for `autogrid4 -p gpf -l glg`: parse, compute on the GPU, write the maps."""
    job = Job(gpf, glg)
    try:
        prob = job.problem()
        ctx = Context(device)
        try:
            maps = ctx.compute(prob, precision)
        finally:
            ctx.close()
        job.write_maps(maps)
        return maps
    except AutoGridError as e:
        job.fail(e.message)
        raise
    finally:
        job.close()
