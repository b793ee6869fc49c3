"""ORACLE — test infrastructure only.

ctypes bindings of ``oracle/refcpu.cpp``, the CPU restatement of RustyFEM's
multifrontal LDLᵀ (src/sparse.rs, src/sparse/indef.rs, ffi/src/lib.rs). The
``oref_*`` C functions have the reference's C-interface signatures
(ffi/src/lib.rs:64-407), so this module reads like a ctypes caller of the
reference library (e.g. OpenFEM's plugin).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "librefcpu.so")

_I64 = ctypes.POINTER(ctypes.c_int64)
_F64 = ctypes.POINTER(ctypes.c_double)
_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "refcpu.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "-B" if force else "-s"], check=True, stdout=subprocess.DEVNULL)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        sz = ctypes.c_size_t
        sig = {
            "oref_set_threads": (None, [ctypes.c_int]),
            "oref_sort_unstable_keys": (None, [_I64, sz, ctypes.c_long, _I64]),
            "oref_threads": (ctypes.c_int, []),
            "oref_uses_fma": (ctypes.c_int, []),
            "oref_factor": (vp, [sz, sz, _I64, _F64, _I64, _I64, _F64, _F64, _I64]),
            "oref_factor_indef": (vp, [sz, sz, _I64, _F64, _I64, _I64, _F64, _I64, _I64]),
            "oref_factor_unsym": (vp, [sz, sz, _I64, _F64, _I64, _I64, _F64, _I64]),
            "oref_lu_delayed": (ctypes.c_int64, [vp]),
            "oref_inertia": (ctypes.c_int32, [vp, _I64]),
            "oref_solve": (ctypes.c_int32, [vp, sz, _F64]),
            "oref_info": (None, [vp, _F64]),
            "oref_order": (None, [vp, _I64]),
            "oref_free": (None, [vp]),
            "oref_handle_nfronts": (sz, [vp]),
            "oref_handle_fronts": (None, [vp, _I64]),
            "oref_analyse": (vp, [sz, _F64, _I64, _I64, _I64, sz]),
            "oref_sym_free": (None, [vp]),
            "oref_sym_n": (sz, [vp]),
            "oref_sym_nfronts": (sz, [vp]),
            "oref_sym_work": (ctypes.c_double, [vp]),
            "oref_sym_factor_size": (sz, [vp]),
            "oref_sym_total_rows": (sz, [vp]),
            "oref_sym_fronts": (None, [vp, _I64]),
            "oref_sym_first_dof": (None, [vp, _I64]),
            "oref_sym_rows": (None, [vp, _I64]),
            "oref_sym_children": (None, [vp, _I64]),
            "oref_sym_nnz": (sz, [vp]),
            "oref_sym_pattern": (None, [vp, _I64, _I64]),
            "oref_pd_factor": (vp, [vp, _I64, _I64, _F64, _I64]),
            "oref_pd_solve": (None, [vp, _F64]),
            "oref_pd_pivots": (None, [vp, _F64]),
            "oref_pd_free": (None, [vp]),
            "oref_indef_factor": (vp, [vp, _I64, _I64, _F64, ctypes.c_double, _I64]),
            "oref_indef_solve": (None, [vp, _F64]),
            "oref_indef_stats": (None, [vp, _I64]),
            "oref_indef_free": (None, [vp]),
            "oref_sym_matvec": (None, [sz, _I64, _I64, _F64, _F64, _F64]),
            "oref_indef_solve_refined": (None, [vp, sz, _I64, _I64, _F64, _F64]),
            "oref_staged_begin": (vp, [sz, sz, _I64, _F64, _I64, _I64, _F64, sz, _I64]),
            "oref_staged_nparts": (sz, [vp]),
            "oref_staged_part_work": (ctypes.c_double, [vp, sz]),
            "oref_staged_part": (ctypes.c_int32, [vp, sz]),
            "oref_staged_finish": (vp, [vp, _I64]),
            "oref_ke_hex8": (ctypes.c_int32, [_F64, ctypes.c_double, ctypes.c_double, _F64]),
            "oref_assemble": (ctypes.c_int32, [sz, _I64, _I64, sz, sz, _I64, _F64, _F64, _I64]),
            "oref_assemble_hex8": (ctypes.c_int32, [sz, _I64, _I64, sz, _I64, _F64, _F64, ctypes.c_double, _I64,
                                                    _F64, _I64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return None if a is None else a.ctypes.data_as(t)


def sort_unstable_keys(keys, limit: int = -1) -> np.ndarray:
    """The indices 0..n-1 in the order the restated slice::sort_unstable_by leaves
    them when sorting by ``keys`` (src/sparse.rs:108)."""
    k = np.ascontiguousarray(keys, np.int64)
    out = np.zeros(len(k), np.int64)
    lib().oref_sort_unstable_keys(_p(k, _I64), len(k), limit, _p(out, _I64))
    return out


def set_threads(t: int) -> None:
    lib().oref_set_threads(int(t))


def threads() -> int:
    return lib().oref_threads()


# ---------------------------------------------------------------------------
# The C interface (ffi/src/lib.rs), restated
# ---------------------------------------------------------------------------
class Handle:
    """A factor handle of the oracle's C interface."""

    def __init__(self, ptr, n, kind):
        self.ptr = ptr
        self.n = n
        self.kind = kind

    def solve(self, b: np.ndarray) -> np.ndarray:
        """Solves K X = B for B of shape (n,) or (nrhs, n) (each RHS contiguous); returns X."""
        x = np.array(b, dtype=np.float64, order="C", copy=True)
        nrhs = 1 if x.ndim == 1 else x.shape[0]
        rc = lib().oref_solve(self.ptr, nrhs, _p(x, _F64))
        if rc != 0:
            raise RuntimeError("oref_solve failed")
        return x

    def info(self):
        out = np.zeros(2)
        lib().oref_info(self.ptr, _p(out, _F64))
        return float(out[0]), int(out[1])

    def order(self):
        out = np.zeros(self.n, np.int64)
        lib().oref_order(self.ptr, _p(out, _I64))
        return out

    def inertia(self):
        out = np.zeros(3, np.int64)
        rc = lib().oref_inertia(self.ptr, _p(out, _I64))
        return None if rc != 0 else tuple(int(v) for v in out)

    def fronts(self) -> np.ndarray:
        nf = lib().oref_handle_nfronts(self.ptr)
        out = np.zeros((nf, 4), np.int64)
        lib().oref_handle_fronts(self.ptr, _p(out, _I64))
        return out

    def free(self):
        if self.ptr:
            lib().oref_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _csc_args(model):
    return (model.n, model.nn, _p(np.ascontiguousarray(model.loc, np.int64), _I64),
            _p(np.ascontiguousarray(model.coords, np.float64), _F64),
            _p(np.ascontiguousarray(model.indptr, np.int64), _I64),
            _p(np.ascontiguousarray(model.indices, np.int64), _I64),
            _p(np.ascontiguousarray(model.data, np.float64), _F64))


def factor(model, want_d: bool = False):
    """rustyfem_factor (ffi/src/lib.rs:64-97): returns (handle or None, err_dof, d)."""
    keep = [np.ascontiguousarray(a) for a in (model.loc, model.coords, model.indptr, model.indices, model.data)]
    err = np.zeros(1, np.int64)
    d = np.zeros(model.n) if want_d else None
    ptr = lib().oref_factor(*_csc_args(model), _p(d, _F64), _p(err, _I64))
    del keep
    if not ptr:
        return None, int(err[0]), None
    return Handle(ptr, model.n, "pd"), -1, d


class StagedFactor:
    """rustyfem_factor cut into consecutive parts (``oref_staged_*``): ``begin`` runs the
    analysis, ``part(p)`` for p = 0 … nparts-1 finishes the subtrees of one range of
    fronts (equal shares of the flops), ``finish`` returns the :class:`Handle`. The factor
    is bit for bit the one :func:`factor` computes; the parts let a benchmark time one
    whole factorization in slices of bounded length."""

    def __init__(self, model, nparts: int):
        self._keep = [np.ascontiguousarray(a) for a in (model.loc, model.coords, model.indptr, model.indices,
                                                       model.data)]
        self.model = model
        err = np.zeros(1, np.int64)
        self.ptr = lib().oref_staged_begin(*_csc_args(model), int(nparts), _p(err, _I64))
        if not self.ptr:
            raise RuntimeError(f"oracle analysis failed (err_dof {int(err[0])})")
        self.nparts = int(lib().oref_staged_nparts(self.ptr))

    def part_work(self, p: int) -> float:
        return float(lib().oref_staged_part_work(self.ptr, p))

    def part(self, p: int) -> bool:
        return lib().oref_staged_part(self.ptr, int(p)) == 0

    def finish(self):
        err = np.zeros(1, np.int64)
        ptr = lib().oref_staged_finish(self.ptr, _p(err, _I64))
        self.ptr = None
        if not ptr:
            return None, int(err[0])
        return Handle(ptr, self.model.n, "pd"), -1


def factor_indef(model):
    """rustyfem_factor_indef (ffi/src/lib.rs:273-290): returns (handle or None, err_dof, inertia)."""
    err = np.zeros(1, np.int64)
    ine = np.zeros(3, np.int64)
    ptr = lib().oref_factor_indef(*_csc_args(model), _p(ine, _I64), _p(err, _I64))
    if not ptr:
        return None, int(err[0]), None
    return Handle(ptr, model.n, "indef"), -1, tuple(int(v) for v in ine)


def factor_unsym(model):
    """rustyfem_factor_unsym (ffi/src/lib.rs:300-311): multifrontal LU of a matrix given with both
    triangles. Returns (handle or None, err_dof, delayed pivots)."""
    err = np.zeros(1, np.int64)
    ptr = lib().oref_factor_unsym(*_csc_args(model), _p(err, _I64))
    if not ptr:
        return None, int(err[0]), None
    return Handle(ptr, model.n, "lu"), -1, int(lib().oref_lu_delayed(ptr))


# ---------------------------------------------------------------------------
# Engine-level API: analyse / pattern / factor / solve (src/sparse.rs)
# ---------------------------------------------------------------------------
class Symbolic:
    """``sparse::analyse_with_leaf`` on a node graph (src/sparse.rs:167-232)."""

    def __init__(self, graph, leaf: int = 48):
        self.graph = graph
        coords = np.ascontiguousarray(graph.coords, np.float64)
        self.ptr = lib().oref_analyse(len(graph.ndof), _p(coords, _F64), _p(graph.adj_ptr, _I64),
                                      _p(graph.adj_idx, _I64), _p(graph.ndof, _I64), leaf)
        L = lib()
        self.n = L.oref_sym_n(self.ptr)
        self.nfronts = L.oref_sym_nfronts(self.ptr)

    def work(self) -> float:
        return lib().oref_sym_work(self.ptr)

    def factor_size(self) -> int:
        return lib().oref_sym_factor_size(self.ptr)

    def fronts(self) -> np.ndarray:
        out = np.zeros((self.nfronts, 4), np.int64)
        lib().oref_sym_fronts(self.ptr, _p(out, _I64))
        return out

    def first_dof(self) -> np.ndarray:
        out = np.zeros(len(self.graph.ndof), np.int64)
        lib().oref_sym_first_dof(self.ptr, _p(out, _I64))
        return out

    def rows(self) -> np.ndarray:
        out = np.zeros(lib().oref_sym_total_rows(self.ptr), np.int64)
        lib().oref_sym_rows(self.ptr, _p(out, _I64))
        return out

    def children(self) -> np.ndarray:
        nch = int(self.fronts()[:, 3].sum())
        out = np.zeros(nch, np.int64)
        lib().oref_sym_children(self.ptr, _p(out, _I64))
        return out

    def pattern(self):
        nnz = lib().oref_sym_nnz(self.ptr)
        colptr = np.zeros(self.n + 1, np.int64)
        rowidx = np.zeros(nnz, np.int64)
        lib().oref_sym_pattern(self.ptr, _p(colptr, _I64), _p(rowidx, _I64))
        return colptr, rowidx

    def pd_factor(self, colptr, rowidx, val):
        err = np.zeros(1, np.int64)
        ptr = lib().oref_pd_factor(self.ptr, _p(colptr, _I64), _p(rowidx, _I64), _p(val, _F64), _p(err, _I64))
        return (PdFactor(ptr) if ptr else None), int(err[0])

    def indef_factor(self, colptr, rowidx, val, threshold: float = 0.01):
        err = np.zeros(1, np.int64)
        ptr = lib().oref_indef_factor(self.ptr, _p(colptr, _I64), _p(rowidx, _I64), _p(val, _F64), threshold,
                                      _p(err, _I64))
        return (IndefFactor(ptr) if ptr else None), int(err[0])

    def __del__(self):
        try:
            lib().oref_sym_free(self.ptr)
        except Exception:
            pass


class PdFactor:
    def __init__(self, ptr):
        self.ptr = ptr

    def solve(self, x: np.ndarray) -> np.ndarray:
        y = np.array(x, dtype=np.float64, copy=True)
        lib().oref_pd_solve(self.ptr, _p(y, _F64))
        return y

    def pivots(self, n: int) -> np.ndarray:
        d = np.zeros(n)
        lib().oref_pd_pivots(self.ptr, _p(d, _F64))
        return d

    def __del__(self):
        try:
            lib().oref_pd_free(self.ptr)
        except Exception:
            pass


class IndefFactor:
    def __init__(self, ptr):
        self.ptr = ptr

    def solve(self, x: np.ndarray) -> np.ndarray:
        y = np.array(x, dtype=np.float64, copy=True)
        lib().oref_indef_solve(self.ptr, _p(y, _F64))
        return y

    def stats(self) -> dict:
        out = np.zeros(6, np.int64)
        lib().oref_indef_stats(self.ptr, _p(out, _I64))
        return dict(neg=int(out[0]), zero=int(out[1]), pos=int(out[2]), delayed=int(out[3]),
                    two_by_two=int(out[4]), factor_size=int(out[5]))

    def __del__(self):
        try:
            lib().oref_indef_free(self.ptr)
        except Exception:
            pass


def to_internal(model, sym: Symbolic):
    """The lower CSC of ``model`` (node-major caller numbering, graph blocks = free nodes in order)
    mapped into the internal numbering of ``sym`` (src/fem/assembly.rs:289-301 + SystemMatrix::add)."""
    colptr, rowidx = sym.pattern()
    fd = sym.first_dof()
    # caller DOF -> block and slot: blocks are the nodes carrying DOFs, in order
    nodes, first = np.unique(model.loc, return_index=True)
    block_of_node = {int(v): i for i, v in enumerate(nodes)}
    blk = np.array([block_of_node[int(v)] for v in model.loc], np.int64)
    slot = np.arange(model.n) - first[blk]
    eq = fd[blk] + slot
    val = np.zeros(len(rowidx))
    cols = np.repeat(np.arange(model.n), np.diff(model.indptr))
    qr = eq[model.indices]
    qc = eq[cols]
    r = np.maximum(qr, qc)
    c = np.minimum(qr, qc)
    # position of (r, c) in the pattern: rows are sorted within each column
    for i in range(len(r)):
        lo, hi = colptr[c[i]], colptr[c[i] + 1]
        pos = lo + np.searchsorted(rowidx[lo:hi], r[i])
        val[pos] += model.data[i]
    return colptr, rowidx, val, eq


def sym_matvec(colptr, rowidx, val, x):
    y = np.zeros_like(x)
    n = len(colptr) - 1
    lib().oref_sym_matvec(n, _p(colptr, _I64), _p(rowidx, _I64), _p(val, _F64), _p(x, _F64), _p(y, _F64))
    return y


def ke_hex8(x: np.ndarray, E: float, nu: float) -> np.ndarray:
    """The C3D8 element matrix (24×24) at node coordinates x (8×3): src/elements/continuum3d.rs:39-131."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(24)
    ke = np.zeros(576)
    if lib().oref_ke_hex8(_p(x, _F64), float(E), float(nu), _p(ke, _F64)) != 0:
        raise ValueError("distorted element (det J <= 0 at an integration point)")
    return ke.reshape(24, 24)


def assemble(colptr, rowidx, edof: np.ndarray, ke: np.ndarray) -> np.ndarray:
    """SystemMatrix::zero + the symmetric element loop of src/fem/assembly.rs:388-412: the values of
    the lower CSC (colptr, rowidx) from element matrices ke (nelem, nd, nd) and equation maps
    edof (nelem, nd; -1 = none)."""
    n = len(colptr) - 1
    nelem, nd = edof.shape
    edof = np.ascontiguousarray(edof, dtype=np.int64)
    ke = np.ascontiguousarray(ke, dtype=np.float64)
    val = np.zeros(int(colptr[-1]))
    bad = np.zeros(2, np.int64)
    if lib().oref_assemble(n, _p(colptr, _I64), _p(rowidx, _I64), nelem, nd, _p(edof, _I64), _p(ke, _F64),
                           _p(val, _F64), _p(bad, _I64)) != 0:
        raise KeyError(f"entry ({bad[0]}, {bad[1]}) missing in the pattern")
    return val


def assemble_hex8(colptr, rowidx, conn, xyz, emod, nu: float, edof) -> np.ndarray:
    """`internal`'s tangent assembly of a C3D8 mesh (element matrices in parallel blocks of 8192,
    added in element order): the lower CSC values."""
    n = len(colptr) - 1
    conn = np.ascontiguousarray(conn, dtype=np.int64)
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    emod = np.ascontiguousarray(emod, dtype=np.float64)
    edof = np.ascontiguousarray(edof, dtype=np.int64)
    val = np.zeros(int(colptr[-1]))
    bad = np.zeros(2, np.int64)
    r = lib().oref_assemble_hex8(n, _p(colptr, _I64), _p(rowidx, _I64), len(conn), _p(conn, _I64), _p(xyz, _F64),
                                 _p(emod, _F64), float(nu), _p(edof, _I64), _p(val, _F64), _p(bad, _I64))
    if r == -1:
        raise KeyError(f"entry ({bad[0]}, {bad[1]}) missing in the pattern")
    if r == -2:
        raise ValueError(f"element {bad[0]} is distorted")
    return val
