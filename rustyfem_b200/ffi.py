"""ctypes bindings of librustyfem_gpu.so (include/rustyfem_gpu.h).

The module mirrors how RustyFEM's C interface is used from Python (the
reference's ctypes callers): ``factor`` / ``factor_indef`` return a handle or
the caller's DOF of the failing pivot, ``Handle.solve`` solves in place for
one or many right-hand sides, ``info`` / ``order`` / ``inertia`` report on the
factorization (ffi/src/lib.rs:57-407). The numeric phase runs on the GPU; the
library refuses to factor without one (there is no CPU path).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _build

_I64 = ctypes.POINTER(ctypes.c_int64)
_F64 = ctypes.POINTER(ctypes.c_double)
_lib = None

FP64 = 0
MIXED = 1
AUTO = 2

# every symbol the header declares (checked by the tests)
EXPORTS = [
    "rustyfem_factor", "rustyfem_factor_indef", "rustyfem_factor_unsym", "rustyfem_inertia", "rustyfem_solve",
    "rustyfem_info", "rustyfem_order", "rustyfem_free",
    "rfg_factor_ex", "rfg_batch_factor", "rfg_refactor", "rfg_refactor_device", "rfg_solve_ex", "rfg_solve_device", "rfg_solve_device_noalloc", "rfg_tune_report", "rfg_tune_report_ex", "rfg_release_cached_memory", "rfg_stream",
    "rfg_set_profiling", "rfg_factor_stats_get", "rfg_handle_nfronts",
    "rfg_handle_fronts", "rfg_last_error", "rfg_device_count", "rfg_selftest_reciprocal",
    "rfg_selftest_sort_unstable",
    "rfg_matrix_prepare", "rfg_matrix_n", "rfg_matrix_first_dof", "rfg_matrix_zero", "rfg_matrix_add",
    "rfg_matrix_add_many", "rfg_matrix_factor", "rfg_matrix_solve", "rfg_matrix_free", "rfg_matrix_nnz",
    "rfg_matrix_values", "rfg_assembly_prepare", "rfg_assembly_set", "rfg_assembly_set_device",
    "rfg_assembly_hex8", "rfg_assembly_times", "rfg_assembly_contributions", "rfg_assembly_free",
    "rfg_sym_analyse", "rfg_sym_n", "rfg_sym_nfronts", "rfg_sym_work", "rfg_sym_factor_size",
    "rfg_sym_total_rows", "rfg_sym_fronts", "rfg_sym_first_dof", "rfg_sym_rows", "rfg_sym_children",
    "rfg_sym_nnz", "rfg_sym_pattern", "rfg_sym_plan_stats", "rfg_sym_plan_flops", "rfg_sym_free",
]


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("leaf", ctypes.c_int32), ("refine_max_iter", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("refine_tol", ctypes.c_double)]


FLAG_NO_TENSOR_CORES = 1
FLAG_AUTOTUNE = 2


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("launches", ctypes.c_int32), ("backward_error", ctypes.c_double),
                ("rel_residual", ctypes.c_double), ("t_solve_ms", ctypes.c_double)]


class FactorStats(ctypes.Structure):
    _fields_ = [("work", ctypes.c_double), ("factor_size", ctypes.c_double), ("t_analyse_ms", ctypes.c_double),
                ("t_factor_ms", ctypes.c_double), ("nfronts", ctypes.c_int64), ("nlevels", ctypes.c_int64),
                ("nsteps", ctypes.c_int64), ("launches", ctypes.c_int64), ("panel_bytes", ctypes.c_int64),
                ("update_bytes", ctypes.c_int64), ("largest_k", ctypes.c_int64), ("largest_u", ctypes.c_int64),
                ("schur_ms", ctypes.c_double), ("schur_flops", ctypes.c_double), ("schur_launches", ctypes.c_int64),
                ("h2d_bytes", ctypes.c_int64), ("phase_ms", ctypes.c_double * 7),
                ("tile_cutover_rows", ctypes.c_int64), ("tc_kind", ctypes.c_int64),
                ("outer_tile_n", ctypes.c_int64), ("precision", ctypes.c_int64),
                ("schur_entries", ctypes.c_double), ("schur_opvals", ctypes.c_double),
                ("delayed", ctypes.c_int64)]


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        L = ctypes.CDLL(_build.gpu_library())
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        csc = [sz, sz, _I64, _F64, _I64, _I64, _F64]
        sig = {
            "rustyfem_factor": (vp, csc + [_F64, _I64]),
            "rustyfem_factor_indef": (vp, csc + [_I64, _I64]),
            "rustyfem_factor_unsym": (vp, csc + [_I64]),
            "rustyfem_inertia": (ctypes.c_int32, [vp, _I64]),
            "rustyfem_solve": (ctypes.c_int32, [vp, sz, _F64]),
            "rustyfem_info": (None, [vp, _F64]),
            "rustyfem_order": (None, [vp, _I64]),
            "rustyfem_free": (None, [vp]),
            "rfg_factor_ex": (vp, csc + [ctypes.POINTER(Options), _F64, _I64]),
            "rfg_refactor": (ctypes.c_int64, [vp, _F64]),
            "rfg_batch_factor": (vp, [sz, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.POINTER(_I64), ctypes.POINTER(_F64), ctypes.POINTER(_I64),
                                      ctypes.POINTER(_I64), ctypes.POINTER(_F64), ctypes.POINTER(Options), _I64,
                                      _I64]),
            "rfg_refactor_device": (ctypes.c_int64, [vp, ctypes.c_void_p]),
            "rfg_solve_device": (ctypes.c_int32, [vp, sz, ctypes.c_void_p, ctypes.POINTER(SolveStats)]),
            "rfg_solve_device_noalloc": (ctypes.c_int32, [vp, sz, ctypes.c_void_p]),
            "rfg_tune_report": (sz, [vp, _I64, _F64, sz]),
            "rfg_tune_report_ex": (sz, [vp, _I64, _I64, _F64, sz]),
            "rfg_release_cached_memory": (None, []),
            "rfg_stream": (vp, [vp]),
            "rfg_set_profiling": (None, [vp, ctypes.c_int32]),
            "rfg_solve_ex": (ctypes.c_int32, [vp, sz, _F64, ctypes.POINTER(SolveStats)]),
            "rfg_factor_stats_get": (ctypes.c_int32, [vp, ctypes.POINTER(FactorStats)]),
            "rfg_handle_nfronts": (sz, [vp]),
            "rfg_handle_fronts": (None, [vp, _I64]),
            "rfg_last_error": (ctypes.c_char_p, []),
            "rfg_device_count": (ctypes.c_int32, []),
            "rfg_selftest_reciprocal": (ctypes.c_int32, [_F64, _F64, sz]),
            "rfg_selftest_sort_unstable": (None, [_I64, ctypes.c_int64, ctypes.c_int64, _I64]),
            "rfg_matrix_prepare": (vp, [sz, _F64, _I64, _I64, _I64, ctypes.c_int32, ctypes.c_int32]),
            "rfg_matrix_n": (sz, [vp]),
            "rfg_matrix_first_dof": (None, [vp, _I64]),
            "rfg_matrix_zero": (None, [vp]),
            "rfg_matrix_add": (ctypes.c_int32, [vp, sz, sz, ctypes.c_double]),
            "rfg_matrix_add_many": (ctypes.c_int32, [vp, sz, _I64, _I64, _F64]),
            "rfg_matrix_factor": (ctypes.c_int64, [vp]),
            "rfg_matrix_solve": (ctypes.c_int32, [vp, _F64]),
            "rfg_matrix_free": (None, [vp]),
            "rfg_matrix_nnz": (sz, [vp]),
            "rfg_matrix_values": (ctypes.c_int32, [vp, _F64]),
            "rfg_assembly_prepare": (vp, [vp, sz, sz, _I64]),
            "rfg_assembly_set": (ctypes.c_int32, [vp, _F64]),
            "rfg_assembly_set_device": (ctypes.c_int32, [vp, vp]),
            "rfg_assembly_hex8": (ctypes.c_int64, [vp, sz, _F64, _I64, _F64, ctypes.c_double]),
            "rfg_assembly_times": (None, [vp, _F64]),
            "rfg_assembly_contributions": (sz, [vp]),
            "rfg_assembly_free": (None, [vp]),
            "rfg_sym_analyse": (vp, [sz, _F64, _I64, _I64, _I64, ctypes.c_int32]),
            "rfg_sym_n": (sz, [vp]),
            "rfg_sym_nfronts": (sz, [vp]),
            "rfg_sym_work": (ctypes.c_double, [vp]),
            "rfg_sym_factor_size": (sz, [vp]),
            "rfg_sym_total_rows": (sz, [vp]),
            "rfg_sym_fronts": (None, [vp, _I64]),
            "rfg_sym_first_dof": (None, [vp, _I64]),
            "rfg_sym_rows": (None, [vp, _I64]),
            "rfg_sym_children": (None, [vp, _I64]),
            "rfg_sym_nnz": (sz, [vp]),
            "rfg_sym_pattern": (None, [vp, _I64, _I64]),
            "rfg_sym_plan_stats": (None, [vp, _I64]),
            "rfg_sym_plan_flops": (None, [vp, ctypes.c_int64, _F64]),
            "rfg_sym_free": (None, [vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def last_error() -> str:
    return lib().rfg_last_error().decode()


def device_count() -> int:
    return int(lib().rfg_device_count())


def sort_unstable_keys(keys, limit: int = -1) -> np.ndarray:
    """The indices 0..n-1 in the order the symbolic stage's coordinate sort (Rust's
    slice::sort_unstable_by, src/sparse.rs:108) leaves them when sorting by ``keys``."""
    k = np.ascontiguousarray(keys, np.int64)
    out = np.zeros(len(k), np.int64)
    lib().rfg_selftest_sort_unstable(_p(k, _I64), len(k), limit, _p(out, _I64))
    return out


class FactorError(RuntimeError):
    """The factorization failed: ``dof`` is the caller's DOF of the failing pivot, or -1."""

    def __init__(self, dof: int, msg: str):
        super().__init__(f"{msg} (DOF {dof})")
        self.dof = dof


class Handle:
    """A factorization of the C interface (``RustyfemHandle*``)."""

    def __init__(self, ptr, n: int, kind: str):
        self.ptr = ptr
        self.n = n
        self.kind = kind

    def solve(self, b: np.ndarray, stats: bool = False):
        """Solves K X = B for B of shape (n,) or (nrhs, n); returns X (and the solve
        statistics with ``stats=True``). rustyfem_solve, ffi/src/lib.rs:337-371."""
        x = np.array(b, dtype=np.float64, order="C", copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[0]
        if stats:
            st = SolveStats()
            rc = lib().rfg_solve_ex(self.ptr, nrhs, _p(x, _F64), ctypes.byref(st))
        else:
            rc = lib().rustyfem_solve(self.ptr, nrhs, _p(x, _F64))
        if rc != 0:
            raise RuntimeError("rustyfem_solve failed: " + last_error())
        if stats:
            return x, dict(iterations=st.iterations, backward_error=st.backward_error,
                           rel_residual=st.rel_residual, t_solve_ms=st.t_solve_ms, launches=st.launches)
        return x

    def solve_inplace(self, b: np.ndarray) -> None:
        """rustyfem_solve on a caller buffer (contiguous float64, n or nrhs×n)."""
        assert b.dtype == np.float64 and b.flags.c_contiguous
        nrhs = 1 if b.ndim == 1 else b.shape[0]
        if lib().rustyfem_solve(self.ptr, nrhs, _p(b, _F64)) != 0:
            raise RuntimeError("rustyfem_solve failed: " + last_error())

    def refactor_device(self, data_ptr: int) -> int:
        """Numeric phase from values already on the device (pointer to nnz float64)."""
        return int(lib().rfg_refactor_device(self.ptr, ctypes.c_void_p(data_ptr)))

    def solve_device(self, b_ptr: int, nrhs: int = 1) -> dict:
        """Solves in place for right-hand sides on the device (caller numbering, column-major)."""
        st = SolveStats()
        if lib().rfg_solve_device(self.ptr, nrhs, ctypes.c_void_p(b_ptr), ctypes.byref(st)) != 0:
            raise RuntimeError("rfg_solve_device failed: " + last_error())
        return dict(iterations=st.iterations, backward_error=st.backward_error, rel_residual=st.rel_residual,
                    t_solve_ms=st.t_solve_ms, launches=st.launches)

    def solve_device_noalloc(self, b_ptr: int, nrhs: int = 1) -> None:
        """Solves in place for right-hand sides on the device (caller numbering,
        column-major) through rfg_solve_device_noalloc: no device allocation, no
        refinement, scratch limited to a fixed 16 MiB."""
        if lib().rfg_solve_device_noalloc(self.ptr, nrhs, ctypes.c_void_p(b_ptr)) != 0:
            raise RuntimeError("rfg_solve_device_noalloc failed: " + last_error())

    def stream(self) -> int:
        return int(lib().rfg_stream(self.ptr) or 0)

    def set_profiling(self, level) -> None:
        """0/False off; 1/True an event after every launch (phase_ms, schur_ms); 2 events
        around the 128-tile outer updates only (schur_ms)."""
        lib().rfg_set_profiling(self.ptr, int(level))

    def refactor(self, data: np.ndarray) -> int:
        """New values on the same pattern; -1 on success, else the failing DOF."""
        d = np.ascontiguousarray(data, np.float64)
        return int(lib().rfg_refactor(self.ptr, _p(d, _F64)))

    def info(self):
        out = np.zeros(2)
        lib().rustyfem_info(self.ptr, _p(out, _F64))
        return float(out[0]), int(out[1])

    def order(self):
        out = np.zeros(self.n, np.int64)
        lib().rustyfem_order(self.ptr, _p(out, _I64))
        return out

    def inertia(self):
        out = np.zeros(3, np.int64)
        rc = lib().rustyfem_inertia(self.ptr, _p(out, _I64))
        return None if rc != 0 else tuple(int(v) for v in out)

    def fronts(self) -> np.ndarray:
        nf = lib().rfg_handle_nfronts(self.ptr)
        out = np.zeros((nf, 4), np.int64)
        lib().rfg_handle_fronts(self.ptr, _p(out, _I64))
        return out

    def stats(self) -> dict:
        st = FactorStats()
        lib().rfg_factor_stats_get(self.ptr, ctypes.byref(st))
        out = {k: getattr(st, k) for k, _ in FactorStats._fields_}
        out["phase_ms"] = list(out["phase_ms"])
        return out

    def tune_report(self) -> list:
        """[(cutover rows, numeric-phase ms)] measured by the autotuner (RFG_FLAG_AUTOTUNE)."""
        return [(c, ms) for c, _, ms in self.tune_report_ex()]

    def tune_report_ex(self) -> list:
        """[(cutover rows, outer tile width, numeric-phase ms)] measured by the autotuner."""
        cnt = lib().rfg_tune_report_ex(self.ptr, None, None, None, 0)
        c = np.zeros(cnt, np.int64)
        tn = np.zeros(cnt, np.int64)
        ms = np.zeros(cnt)
        lib().rfg_tune_report_ex(self.ptr, _p(c, _I64), _p(tn, _I64), _p(ms, _F64), cnt)
        return list(zip(c.tolist(), tn.tolist(), ms.tolist()))

    def free(self):
        if self.ptr:
            lib().rustyfem_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _args(model):
    arrs = [np.ascontiguousarray(model.loc, np.int64), np.ascontiguousarray(model.coords, np.float64),
            np.ascontiguousarray(model.indptr, np.int64), np.ascontiguousarray(model.indices, np.int64),
            np.ascontiguousarray(model.data, np.float64)]
    ptrs = [model.n, model.nn, _p(arrs[0], _I64), _p(arrs[1], _F64), _p(arrs[2], _I64), _p(arrs[3], _I64),
            _p(arrs[4], _F64)]
    return arrs, ptrs


def _flags(tensor_cores: bool, autotune: bool) -> int:
    return (0 if tensor_cores else FLAG_NO_TENSOR_CORES) | (FLAG_AUTOTUNE if autotune else 0)


def factor(model, precision: int = FP64, leaf: int = 0, want_d: bool = False, refine_max_iter: int = -1,
           refine_tol: float = 0.0, raise_on_error: bool = False, tensor_cores: bool = True, autotune: bool = False):
    """rustyfem_factor (or rfg_factor_ex with options). Returns (handle or None, err_dof, d)."""
    keep, ptrs = _args(model)
    err = np.zeros(1, np.int64)
    d = np.zeros(model.n) if want_d else None
    if precision == FP64 and leaf == 0 and refine_max_iter < 0 and refine_tol == 0.0 and not autotune:
        ptr = lib().rustyfem_factor(*ptrs, _p(d, _F64), _p(err, _I64))
    else:
        o = Options(precision, leaf, refine_max_iter, _flags(tensor_cores, autotune), refine_tol)
        ptr = lib().rfg_factor_ex(*ptrs, ctypes.byref(o), _p(d, _F64), _p(err, _I64))
    del keep
    if not ptr:
        if raise_on_error:
            raise FactorError(int(err[0]), last_error())
        return None, int(err[0]), None
    return Handle(ptr, model.n, "pd"), -1, d


class BatchHandle(Handle):
    """A batched factorization of many models (rfg_batch_factor): DOFs stacked model after model."""

    def __init__(self, ptr, sizes):
        self.sizes = list(sizes)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        super().__init__(ptr, int(self.offsets[-1]), "batch")

    def stack(self, per_model):
        """Per-model arrays of shape (n_i,) or (nrhs, n_i) -> the stacked (nrhs, Σ n_i) layout."""
        per_model = [np.asarray(a, np.float64) for a in per_model]
        if per_model[0].ndim == 1:
            return np.concatenate(per_model)
        return np.ascontiguousarray(np.concatenate(per_model, axis=1))

    def split(self, stacked):
        o = self.offsets
        if stacked.ndim == 1:
            return [stacked[o[i]:o[i + 1]] for i in range(len(self.sizes))]
        return [stacked[:, o[i]:o[i + 1]] for i in range(len(self.sizes))]

    def solve_models(self, per_model, stats: bool = False):
        res = self.solve(self.stack(per_model), stats=stats)
        if stats:
            return self.split(res[0]), res[1]
        return self.split(res)


def factor_batch(models, precision: int = FP64, leaf: int = 0, refine_max_iter: int = -1, refine_tol: float = 0.0,
                 tensor_cores: bool = True, autotune: bool = False):
    """rfg_batch_factor: returns (BatchHandle or None, err_model, err_dof)."""
    k = len(models)
    keep = []

    def arr(vals, ctype, dtype):
        arrays = [np.ascontiguousarray(v, dtype) for v in vals]
        keep.extend(arrays)
        ptrs = (ctypes.POINTER(ctype) * k)(*[a.ctypes.data_as(ctypes.POINTER(ctype)) for a in arrays])
        keep.append(ptrs)
        return ptrs

    n = (ctypes.c_size_t * k)(*[m.n for m in models])
    nn = (ctypes.c_size_t * k)(*[m.nn for m in models])
    loc = arr([m.loc for m in models], ctypes.c_int64, np.int64)
    coords = arr([m.coords for m in models], ctypes.c_double, np.float64)
    ip = arr([m.indptr for m in models], ctypes.c_int64, np.int64)
    ix = arr([m.indices for m in models], ctypes.c_int64, np.int64)
    da = arr([m.data for m in models], ctypes.c_double, np.float64)
    o = Options(precision, leaf, refine_max_iter, _flags(tensor_cores, autotune), refine_tol)
    em = np.zeros(1, np.int64)
    ed = np.zeros(1, np.int64)
    ptr = lib().rfg_batch_factor(k, n, nn, loc, coords, ip, ix, da, ctypes.byref(o), _p(em, _I64), _p(ed, _I64))
    del keep
    if not ptr:
        return None, int(em[0]), int(ed[0])
    return BatchHandle(ptr, [m.n for m in models]), -1, -1


def factor_indef(model):
    """rustyfem_factor_indef. Returns (handle or None, err_dof, inertia)."""
    keep, ptrs = _args(model)
    err = np.zeros(1, np.int64)
    ine = np.zeros(3, np.int64)
    ptr = lib().rustyfem_factor_indef(*ptrs, _p(ine, _I64), _p(err, _I64))
    del keep
    if not ptr:
        return None, int(err[0]), None
    return Handle(ptr, model.n, "indef"), -1, tuple(int(v) for v in ine)


def factor_unsym(model):
    """rustyfem_factor_unsym (multifrontal LU; the matrix with both triangles). Returns (handle or
    None, err_dof, factor statistics of the handle or None)."""
    keep, ptrs = _args(model)
    err = np.zeros(1, np.int64)
    ptr = lib().rustyfem_factor_unsym(*ptrs, _p(err, _I64))
    del keep
    if not ptr:
        return None, int(err[0]), None
    h = Handle(ptr, model.n, "lu")
    return h, -1, h.stats()


class Symbolic:
    """The host symbolic stage alone (rfg_sym_*): no GPU needed."""

    def __init__(self, graph, leaf: int = 48):
        self.graph = graph
        self._coords = np.ascontiguousarray(graph.coords, np.float64)
        self.ptr = lib().rfg_sym_analyse(len(graph.ndof), _p(self._coords, _F64), _p(graph.adj_ptr, _I64),
                                         _p(graph.adj_idx, _I64), _p(graph.ndof, _I64), leaf)
        if not self.ptr:
            raise RuntimeError(last_error())
        self.n = lib().rfg_sym_n(self.ptr)
        self.nfronts = lib().rfg_sym_nfronts(self.ptr)

    def work(self) -> float:
        return lib().rfg_sym_work(self.ptr)

    def factor_size(self) -> int:
        return lib().rfg_sym_factor_size(self.ptr)

    def fronts(self) -> np.ndarray:
        out = np.zeros((self.nfronts, 4), np.int64)
        lib().rfg_sym_fronts(self.ptr, _p(out, _I64))
        return out

    def first_dof(self) -> np.ndarray:
        out = np.zeros(len(self.graph.ndof), np.int64)
        lib().rfg_sym_first_dof(self.ptr, _p(out, _I64))
        return out

    def rows(self) -> np.ndarray:
        out = np.zeros(lib().rfg_sym_total_rows(self.ptr), np.int64)
        lib().rfg_sym_rows(self.ptr, _p(out, _I64))
        return out

    def children(self) -> np.ndarray:
        out = np.zeros(int(self.fronts()[:, 3].sum()), np.int64)
        lib().rfg_sym_children(self.ptr, _p(out, _I64))
        return out

    def pattern(self):
        nnz = lib().rfg_sym_nnz(self.ptr)
        colptr = np.zeros(self.n + 1, np.int64)
        rowidx = np.zeros(nnz, np.int64)
        lib().rfg_sym_pattern(self.ptr, _p(colptr, _I64), _p(rowidx, _I64))
        return colptr, rowidx

    def plan_stats(self) -> dict:
        out = np.zeros(4, np.int64)
        lib().rfg_sym_plan_stats(self.ptr, _p(out, _I64))
        return dict(levels=int(out[0]), steps=int(out[1]), panel_elems=int(out[2]), update_elems=int(out[3]))

    def plan_flops(self, cutover_rows: int = 0) -> dict:
        out = np.zeros(4)
        lib().rfg_sym_plan_flops(self.ptr, cutover_rows, _p(out, _F64))
        return dict(inner=out[0], outer=out[1], outer_128tiles=out[2], tiles_128=int(out[3]))

    def __del__(self):
        try:
            lib().rfg_sym_free(self.ptr)
        except Exception:
            pass


_ = os
