"""The engine-side solver API of RustyFEM (src/solver/api.rs:12-60,
src/solver/mod.rs:12-43), backed by the GPU library.

``select(name)`` returns a ``LinearSolver``; ``prepare(graph)`` runs the symbolic
analysis and returns a zeroed ``SystemMatrix`` that the caller assembles with
``add(r, c, v)`` (r >= c, internal numbering given by ``first_dof``), then
``factor()`` (raises ``NotPositiveDefinite`` with the internal equation, the
reference's ``Err(eq)``) and ``solve(b)`` in place. The matrix is reused
between Newton iterations: ``zero`` → ``add``* → ``factor`` → ``solve``*.

Registered solvers: ``"direct-gpu"`` (FP64, the reference's ``direct``) and
``"direct-gpu-mixed"`` (FP32 factor + FP64 refinement to a backward error of
1e-12).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import ffi
from .workloads import Graph

_I64 = ffi._I64
_F64 = ffi._F64


class NotPositiveDefinite(ArithmeticError):
    """``SystemMatrix::factor`` error: the internal equation of the failing pivot."""

    def __init__(self, eq: int):
        super().__init__(f"the matrix is not positive definite at equation {eq}")
        self.eq = eq


class SystemMatrix:
    """src/solver/api.rs:28-60 for the GPU direct solver."""

    def __init__(self, graph: Graph, leaf: int, precision: int):
        g = graph
        self._coords = np.ascontiguousarray(g.coords, np.float64)
        self._adj_ptr = np.ascontiguousarray(g.adj_ptr, np.int64)
        self._adj_idx = np.ascontiguousarray(g.adj_idx, np.int64)
        self._ndof = np.ascontiguousarray(g.ndof, np.int64)
        self.ptr = ffi.lib().rfg_matrix_prepare(len(g.ndof), ffi._p(self._coords, _F64), ffi._p(self._adj_ptr, _I64),
                                                ffi._p(self._adj_idx, _I64), ffi._p(self._ndof, _I64), leaf,
                                                precision)
        if not self.ptr:
            raise RuntimeError("prepare failed: " + ffi.last_error())
        self._n = ffi.lib().rfg_matrix_n(self.ptr)
        fd = np.zeros(len(g.ndof), np.int64)
        ffi.lib().rfg_matrix_first_dof(self.ptr, ffi._p(fd, _I64))
        self._first_dof = fd

    def n(self) -> int:
        return self._n

    def first_dof(self) -> np.ndarray:
        return self._first_dof

    def zero(self) -> None:
        ffi.lib().rfg_matrix_zero(self.ptr)

    def add(self, r: int, c: int, v: float) -> None:
        if ffi.lib().rfg_matrix_add(self.ptr, r, c, v) != 0:
            raise KeyError(f"internal: entry ({r}, {c}) missing in the pattern")

    def add_many(self, r, c, v) -> None:
        r = np.ascontiguousarray(r, np.int64)
        c = np.ascontiguousarray(c, np.int64)
        v = np.ascontiguousarray(v, np.float64)
        if ffi.lib().rfg_matrix_add_many(self.ptr, len(v), ffi._p(r, _I64), ffi._p(c, _I64), ffi._p(v, _F64)) != 0:
            raise KeyError("internal: an entry is missing in the pattern")

    def add_unsym(self, r: int, c: int, v: float) -> None:
        if r >= c:
            self.add(r, c, v)

    def is_symmetric(self) -> bool:
        return True

    def factor(self) -> None:
        e = ffi.lib().rfg_matrix_factor(self.ptr)
        if e == -2:
            raise RuntimeError(ffi.last_error())
        if e >= 0:
            raise NotPositiveDefinite(int(e))

    def solve(self, b: np.ndarray) -> None:
        """Solves K x = b in place (float64 array of length n)."""
        assert b.dtype == np.float64 and b.flags.c_contiguous and b.size == self._n
        if ffi.lib().rfg_matrix_solve(self.ptr, ffi._p(b, _F64)) != 0:
            raise RuntimeError("solve failed: " + ffi.last_error())

    def inertia(self):
        return None

    def nnz(self) -> int:
        return ffi.lib().rfg_matrix_nnz(self.ptr)

    def values(self) -> np.ndarray:
        """The current values of the lower CSC pattern (internal numbering), host or device assembled."""
        out = np.zeros(self.nnz())
        if ffi.lib().rfg_matrix_values(self.ptr, ffi._p(out, _F64)) != 0:
            raise RuntimeError(ffi.last_error())
        return out

    def assembly(self, edof: np.ndarray) -> "Assembly":
        """The element → equation map of an assembly on the device (``edof``: nelem × nd internal
        equations, -1 = constrained): src/fem/assembly.rs:315-420."""
        return Assembly(self, edof)

    def __del__(self):
        try:
            ffi.lib().rfg_matrix_free(self.ptr)
        except Exception:
            pass


class Assembly:
    """K assembled on the GPU from element matrices, into the values of a ``SystemMatrix``:
    ``zero`` + the element loop of ``internal`` (src/fem/assembly.rs:388-412) in one call."""

    def __init__(self, matrix: SystemMatrix, edof: np.ndarray):
        self._m = matrix  # the matrix outlives the assembly
        edof = np.ascontiguousarray(edof, np.int64)
        assert edof.ndim == 2
        self.nelem, self.nd = edof.shape
        self.ptr = ffi.lib().rfg_assembly_prepare(matrix.ptr, self.nelem, self.nd, ffi._p(edof, _I64))
        if not self.ptr:
            raise KeyError(ffi.last_error())

    def set(self, ke: np.ndarray) -> None:
        """K from element matrices ke (nelem × nd × nd) in host memory."""
        ke = np.ascontiguousarray(ke, np.float64)
        assert ke.size == self.nelem * self.nd * self.nd
        if ffi.lib().rfg_assembly_set(self.ptr, ffi._p(ke, _F64)) != 0:
            raise RuntimeError(ffi.last_error())

    def set_device(self, ke_ptr: int) -> None:
        """K from element matrices at a device address (nelem·nd·nd doubles)."""
        if ffi.lib().rfg_assembly_set_device(self.ptr, ctypes.c_void_p(ke_ptr)) != 0:
            raise RuntimeError(ffi.last_error())

    def hex8(self, xyz: np.ndarray, conn: np.ndarray, emod: np.ndarray, nu: float) -> None:
        """C3D8 linear-elastic element matrices computed on the device, then assembled."""
        xyz = np.ascontiguousarray(xyz, np.float64)
        conn = np.ascontiguousarray(conn, np.int64)
        emod = np.ascontiguousarray(emod, np.float64)
        r = ffi.lib().rfg_assembly_hex8(self.ptr, len(xyz), ffi._p(xyz, _F64), ffi._p(conn, _I64),
                                        ffi._p(emod, _F64), float(nu))
        if r >= 0:
            raise ValueError(ffi.last_error())
        if r == -2:
            raise RuntimeError(ffi.last_error())

    def times(self) -> tuple[float, float]:
        """Device time (ms) of the last element kernel and of the last gather."""
        out = np.zeros(2)
        ffi.lib().rfg_assembly_times(self.ptr, ffi._p(out, _F64))
        return float(out[0]), float(out[1])

    def contributions(self) -> int:
        return ffi.lib().rfg_assembly_contributions(self.ptr)

    def __del__(self):
        try:
            ffi.lib().rfg_assembly_free(self.ptr)
        except Exception:
            pass


class LinearSolver:
    """src/solver/api.rs:21-26."""

    def __init__(self, name: str, precision: int, leaf: int = 48):
        self._name = name
        self.precision = precision
        self.leaf = leaf

    def name(self) -> str:
        return self._name

    def prepare(self, graph: Graph) -> SystemMatrix:
        return SystemMatrix(graph, self.leaf, self.precision)


SOLVERS = [LinearSolver("direct-gpu", ffi.FP64), LinearSolver("direct-gpu-mixed", ffi.MIXED)]


def all_solvers():
    return list(SOLVERS)


def select(name: str | None = None) -> LinearSolver:
    """src/solver/mod.rs:33-43 (default "direct-gpu")."""
    want = (name or "direct-gpu").lower()
    for s in SOLVERS:
        if s.name() == want:
            return s
    raise ValueError(f"solver '{want}' does not exist (registered: {', '.join(s.name() for s in SOLVERS)})")
