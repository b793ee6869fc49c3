"""Synthetic FEM workloads for the multifrontal solver.

Structured linear-elastic meshes assembled by ``csrc/meshgen.cpp`` into the
form the RustyFEM C interface takes (``ffi/src/lib.rs:64-75``): free DOFs in the
caller's numbering, ``loc`` (DOF -> node), node coordinates and the lower
triangle in CSC (``indptr``/``indices``/``data``), plus the engine-side node
graph of ``src/solver/api.rs:12-19`` (coordinates, sorted neighbours, DOFs per
node) and the load vector.

Workloads (sizes as the benchmark configurations name them):
  * ``hex8_cube(n)``   — unit cube of n³ C3D8, steel, x = 0 clamped, fz = -1000 N on x = 1;
  * ``hex20_cube(n)``  — the same with C3D20;
  * ``plate(nx, ny)``  — CPS4 cantilever plate, h = 0.025, t = 0.01, fy = -1000 N on the far edge;
  * ``plate_batch()``  — 512 plates with nx ~ U{20..200} (seeded), ny = max(2, nx // 10);
  * ``chain(...)``     — the 1-D chains of the reference's C-interface test (ffi/src/lib.rs:414-427);
  * ``laplace3d(g)``   — the shifted 7-point Laplacian of examples/solver_bench.rs:89-152.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import os

import numpy as np

from . import _build

_I64 = ctypes.POINTER(ctypes.c_int64)
_F64 = ctypes.POINTER(ctypes.c_double)
_lib = None


def _load():
    global _lib
    if _lib is None:
        path = _build.mesh_library()
        lib = ctypes.CDLL(path)
        for name in ("rfg_mesh_hex8_cube",):
            getattr(lib, name).restype = ctypes.c_void_p
            getattr(lib, name).argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_double, _F64, ctypes.c_double]
        lib.rfg_mesh_hex20_cube.restype = ctypes.c_void_p
        lib.rfg_mesh_hex20_cube.argtypes = [ctypes.c_int64, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.rfg_mesh_plate.restype = ctypes.c_void_p
        lib.rfg_mesh_plate.argtypes = [ctypes.c_int64, ctypes.c_int64] + [ctypes.c_double] * 5
        for name in ("rfg_mesh_n", "rfg_mesh_nn", "rfg_mesh_nnz", "rfg_mesh_nelem", "rfg_mesh_nblocks",
                     "rfg_mesh_adj_nnz"):
            getattr(lib, name).restype = ctypes.c_size_t
            getattr(lib, name).argtypes = [ctypes.c_void_p]
        lib.rfg_mesh_dim.restype = ctypes.c_int64
        lib.rfg_mesh_dim.argtypes = [ctypes.c_void_p]
        lib.rfg_mesh_export.restype = None
        lib.rfg_mesh_export.argtypes = [ctypes.c_void_p, _I64, _F64, _I64, _I64, _F64, _F64]
        lib.rfg_mesh_graph.restype = None
        lib.rfg_mesh_graph.argtypes = [ctypes.c_void_p, _F64, _I64, _I64, _I64]
        lib.rfg_mesh_free.restype = None
        lib.rfg_mesh_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


@dataclasses.dataclass
class Graph:
    """Node graph of ``src/solver/api.rs:12-19``: one block per node with free DOFs."""
    coords: np.ndarray   # (nb, 3) float64
    adj_ptr: np.ndarray  # (nb+1,) int64
    adj_idx: np.ndarray  # neighbours, sorted per block, self excluded
    ndof: np.ndarray     # (nb,) int64


@dataclasses.dataclass
class Model:
    """A symmetric system in the C-interface form plus its node graph."""
    name: str
    n: int
    nn: int
    loc: np.ndarray      # (n,) int64 node of each DOF
    coords: np.ndarray   # (3*nn,) float64
    indptr: np.ndarray   # (n+1,) int64, lower triangle CSC
    indices: np.ndarray  # (nnz,) int64
    data: np.ndarray     # (nnz,) float64
    rhs: np.ndarray      # (n,) float64 (or (nrhs, n) after with_rhs)
    graph: Graph | None = None
    symmetric_storage: str = "lower"  # "lower" or "full" (both triangles)

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def with_rhs(self, nrhs: int, seed: int = 0, scale: float = 1000.0) -> "Model":
        """The same model with ``nrhs`` seeded normal load vectors (column-major n·nrhs)."""
        rng = np.random.default_rng(seed)
        b = rng.standard_normal((nrhs, self.n)) * scale
        return dataclasses.replace(self, rhs=np.ascontiguousarray(b))

    def full(self) -> "Model":
        """The same matrix with both triangles stored (the input the reference's
        positive definite C path needs: ffi/src/lib.rs:216-224 keeps only the entries
        whose internal row is not above the internal column)."""
        import scipy.sparse as sp
        if self.symmetric_storage == "full":
            return self
        low = sp.csc_matrix((self.data, self.indices, self.indptr), shape=(self.n, self.n))
        up = sp.triu(low.T, k=1, format="csc")
        f = (low + up).tocsc()
        f.sort_indices()
        return dataclasses.replace(self, indptr=f.indptr.astype(np.int64), indices=f.indices.astype(np.int64),
                                   data=f.data.astype(np.float64), symmetric_storage="full")

    def dense(self) -> np.ndarray:
        """The full symmetric matrix (small models only)."""
        a = np.zeros((self.n, self.n))
        for c in range(self.n):
            for p in range(self.indptr[c], self.indptr[c + 1]):
                r = self.indices[p]
                a[r, c] += self.data[p]
                if r != c and self.symmetric_storage == "lower":
                    a[c, r] += self.data[p]
        return a

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x for the symmetric matrix stored as its lower triangle."""
        cols = np.repeat(np.arange(self.n), np.diff(self.indptr))
        rows = self.indices
        v = self.data
        y = np.zeros_like(x)
        np.add.at(y, rows, v * x[cols])
        if self.symmetric_storage == "lower":
            off = rows != cols
            np.add.at(y, cols[off], v[off] * x[rows[off]])
        return y


def _from_handle(h, name: str) -> Model:
    lib = _load()
    n = lib.rfg_mesh_n(h)
    nn = lib.rfg_mesh_nn(h)
    nnz = lib.rfg_mesh_nnz(h)
    loc = np.zeros(n, np.int64)
    coords = np.zeros(3 * nn)
    indptr = np.zeros(n + 1, np.int64)
    indices = np.zeros(nnz, np.int64)
    data = np.zeros(nnz)
    rhs = np.zeros(n)
    lib.rfg_mesh_export(h, _p(loc, _I64), _p(coords, _F64), _p(indptr, _I64), _p(indices, _I64), _p(data, _F64),
                        _p(rhs, _F64))
    nb = lib.rfg_mesh_nblocks(h)
    gc = np.zeros((nb, 3))
    ap = np.zeros(nb + 1, np.int64)
    ai = np.zeros(lib.rfg_mesh_adj_nnz(h), np.int64)
    nd = np.zeros(nb, np.int64)
    lib.rfg_mesh_graph(h, _p(gc, _F64), _p(ap, _I64), _p(ai, _I64), _p(nd, _I64))
    lib.rfg_mesh_free(h)
    return Model(name, n, nn, loc, coords, indptr, indices, data, rhs, Graph(gc, ap, ai, nd))


def hex8_cube(n: int, E: float = 210e9, nu: float = 0.3, emod: np.ndarray | None = None,
              fz: float = -1000.0) -> Model:
    """Unit cube of n×n×n C3D8 (src/model.rs:454-500), x = 0 clamped, total fz on the face x = 1."""
    lib = _load()
    if emod is not None:
        emod = np.ascontiguousarray(emod, dtype=np.float64)
        assert emod.size == n ** 3
        h = lib.rfg_mesh_hex8_cube(n, E, nu, _p(emod, _F64), fz)
    else:
        h = lib.rfg_mesh_hex8_cube(n, E, nu, None, fz)
    return _from_handle(h, f"hex8 {n}^3")


@dataclasses.dataclass
class Hex8Mesh:
    """The element form of ``hex8_cube``: what the tangent assembly of src/fem/assembly.rs:315-420
    reads (element connectivity, node coordinates, per-element E), plus the DOF map of
    ``dofmap`` (src/fem/assembly.rs:233-304: blocks = nodes with free DOFs, in node order)."""
    n: int                # elements per edge
    conn: np.ndarray      # (ne, 8) node ids, the C3D8 corner order
    xyz: np.ndarray       # (nn, 3)
    emod: np.ndarray      # (ne,)
    nu: float
    block: np.ndarray     # (nn,) graph block of each node, -1 for clamped nodes

    def edof(self, first_dof: np.ndarray) -> np.ndarray:
        """(ne, 24) internal equations of each element's DOFs (node-major, U1 U2 U3), -1 = clamped:
        dm.eq of src/fem/assembly.rs:289-301 for the solver's first_dof."""
        b = self.block[self.conn]                        # (ne, 8)
        fd = np.where(b >= 0, first_dof[np.maximum(b, 0)], -1)
        eq = fd[:, :, None] + np.arange(3)[None, None, :]
        eq = np.where(b[:, :, None] >= 0, eq, -1)
        return np.ascontiguousarray(eq.reshape(len(self.conn), 24), dtype=np.int64)


def hex8_mesh(n: int, E: float = 210e9, nu: float = 0.3, emod: np.ndarray | None = None) -> Hex8Mesh:
    """The mesh of ``hex8_cube(n)`` (src/model.rs:454-500: nodes x fastest, elements x fastest,
    x = 0 clamped) as arrays."""
    npt = n + 1
    k, j, i = np.meshgrid(np.arange(npt), np.arange(npt), np.arange(npt), indexing="ij")
    xyz = np.stack([i.ravel() / n, j.ravel() / n, k.ravel() / n], axis=1).astype(np.float64)
    ek, ej, ei = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ek, ej, ei = ek.ravel(), ej.ravel(), ei.ravel()

    def nid(a, b, c):
        return (c * npt + b) * npt + a

    conn = np.stack([nid(ei, ej, ek), nid(ei + 1, ej, ek), nid(ei + 1, ej + 1, ek), nid(ei, ej + 1, ek),
                     nid(ei, ej, ek + 1), nid(ei + 1, ej, ek + 1), nid(ei + 1, ej + 1, ek + 1),
                     nid(ei, ej + 1, ek + 1)], axis=1).astype(np.int64)
    free = i.ravel() != 0
    block = np.full(npt ** 3, -1, np.int64)
    block[free] = np.arange(int(free.sum()))
    em = np.full(n ** 3, float(E)) if emod is None else np.ascontiguousarray(emod, dtype=np.float64)
    return Hex8Mesh(n, np.ascontiguousarray(conn), xyz, em, float(nu), block)


def skew_perturbed(model: Model, alpha: float, seed: int = 0) -> Model:
    """An unsymmetric matrix with the pattern of ``model``: A + α·max|diag A|·S with S skew-symmetric
    (S_rc = −S_cr standard normal on the off-diagonal pattern), the kind of tangent that friction or
    follower loads give (src/sparse/lu.rs:1-3). For α of order 10 and more the diagonal fails the LU
    threshold test in places and pivots are delayed; A's symmetric part keeps the matrix regular."""
    import scipy.sparse as sp

    m = model.full()
    A = sp.csc_matrix((m.data, m.indices, m.indptr), shape=(m.n, m.n))
    rng = np.random.default_rng(seed)
    U = sp.triu(A, k=1).tocoo()
    vals = rng.standard_normal(U.nnz) * alpha * float(np.abs(A.diagonal()).max())
    S = sp.coo_matrix((vals, (U.row, U.col)), shape=A.shape)
    B = (A + S - S.T).tocsc()
    B.sort_indices()
    return Model(m.name + f" skew {alpha:g}", m.n, m.nn, m.loc, m.coords, B.indptr.astype(np.int64),
                 B.indices.astype(np.int64), B.data.astype(np.float64), m.rhs, None, "full")


def log_uniform_moduli(n: int, lo: float = 1e3, hi: float = 1e9, seed: int = 0) -> np.ndarray:
    """Per-element E = 10^U(log10 lo, log10 hi) from numpy's PCG64 with ``seed`` (element order x fastest)."""
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(math.log10(lo), math.log10(hi), n ** 3)


def hex20_cube(n: int, E: float = 210e9, nu: float = 0.3, fz: float = -1000.0) -> Model:
    """Unit cube of n×n×n C3D20 (serendipity), x = 0 clamped, total fz on the face x = 1."""
    h = _load().rfg_mesh_hex20_cube(n, E, nu, fz)
    return _from_handle(h, f"hex20 {n}^3")


def plate(nx: int, ny: int, h: float = 0.025, t: float = 0.01, E: float = 210e9, nu: float = 0.3,
          fy: float = -1000.0) -> Model:
    """CPS4 cantilever plate of nx×ny elements (src/model.rs:397-451), x = 0 edge clamped, fy on the far edge."""
    hd = _load().rfg_mesh_plate(nx, ny, h, t, E, nu, fy)
    return _from_handle(hd, f"plate {nx}x{ny}")


def plate_sizes(count: int = 512, seed: int = 0, lo: int = 20, hi: int = 200) -> list[tuple[int, int]]:
    """Seeded plate sizes: nx ~ U{lo..hi}, ny = max(2, nx // 10)."""
    rng = np.random.default_rng(seed)
    nxs = rng.integers(lo, hi + 1, size=count)
    return [(int(nx), max(2, int(nx) // 10)) for nx in nxs]


def plate_batch(count: int = 512, seed: int = 0, nrhs: int = 8) -> list[Model]:
    """``count`` plates of seeded length with ``nrhs`` seeded normal load vectors each."""
    out = []
    for i, (nx, ny) in enumerate(plate_sizes(count, seed)):
        m = plate(nx, ny)
        out.append(m.with_rhs(nrhs, seed=seed * 100003 + i) if nrhs > 0 else m)
    return out


def chain(n: int, diag, off) -> Model:
    """n-DOF chain with one DOF per node on the x axis, CSC with both triangles (ffi/src/lib.rs:414-427)."""
    indptr = [0]
    indices = []
    data = []
    for c in range(n):
        for r in range(max(c - 1, 0), min(c + 2, n)):
            indices.append(r)
            data.append(diag(c) if r == c else off(r, c))
        indptr.append(len(indices))
    coords = np.zeros(3 * n)
    coords[0::3] = np.arange(n, dtype=np.float64)
    return Model(f"chain {n}", n, n, np.arange(n, dtype=np.int64), coords, np.array(indptr, np.int64),
                 np.array(indices, np.int64), np.array(data, np.float64), np.zeros(n), symmetric_storage="full")


def laplace3d(g: int, sigma: float) -> tuple[Model, int]:
    """7-point Laplacian on g³ nodes shifted by sigma (lower CSC) and its analytic number of
    eigenvalues below sigma (examples/solver_bench.rs:89-141)."""
    nn = g * g * g
    idx = np.arange(nn).reshape(g, g, g)  # [k, j, i]
    coords = np.zeros((nn, 3))
    kk, jj, ii = np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij")
    coords[:, 0] = ii.ravel()
    coords[:, 1] = jj.ravel()
    coords[:, 2] = kk.ravel()
    indptr = [0]
    indices = []
    data = []
    for v in range(nn):
        i, j, k = v % g, (v // g) % g, v // (g * g)
        indices.append(v)
        data.append(6.0 - sigma)
        nb = []
        if i + 1 < g:
            nb.append(v + 1)
        if j + 1 < g:
            nb.append(v + g)
        if k + 1 < g:
            nb.append(v + g * g)
        for w in sorted(nb):
            indices.append(w)
            data.append(-1.0)
        indptr.append(len(indices))
    c = 2.0 * np.cos(np.arange(1, g + 1) * np.pi / (g + 1))
    lam = 6.0 - (c[:, None, None] + c[None, :, None] + c[None, None, :])
    below = int(np.count_nonzero(lam < sigma))
    return Model(f"laplace {g}^3", nn, nn, np.arange(nn, dtype=np.int64), coords.ravel(), np.array(indptr, np.int64),
                 np.array(indices, np.int64), np.array(data), np.zeros(nn)), below


def laplace_sigma(g: int) -> float:
    """sigma midway between two distinct eigenvalues near the 10 % quantile (examples/solver_bench.rs:124-140)."""
    c = 2.0 * np.cos(np.arange(1, g + 1) * np.pi / (g + 1))
    lam = np.sort((6.0 - (c[:, None, None] + c[None, :, None] + c[None, None, :])).ravel())
    q = lam.size // 10
    while lam[q + 1] - lam[q] < 1e-9:
        q += 1
    return 0.5 * (lam[q] + lam[q + 1])


_ = os  # the module path helpers live in _build
