"""The GPU indefinite LDLᵀ (rustyfem_factor_indef) against the reference's known
answers and the oracle: inertia, the counts of delayed pivots and 2×2 blocks,
and the solution (relative error 1e-10)."""
import json
import os

import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")


def known():
    with open(GOLD) as f:
        return json.load(f)


def test_chain_inertia_residual(gpu):
    """ffi/src/lib.rs:429-456."""
    k = known()["chain"]
    n, sigma = k["n"], k["sigma"]
    m = W.chain(n, lambda c: 2.0 - sigma, lambda r, c: -1.0)
    h, err, ine = ffi.factor_indef(m)
    assert h is not None, ffi.last_error()
    assert list(ine) == k["inertia"]
    assert h.inertia() == tuple(k["inertia"])
    b = np.sin(np.arange(n) * 0.3)
    x = h.solve(b)
    assert np.max(np.abs(m.dense() @ x - b)) < k["residual_tol"]


def test_chain_singular_dof(gpu):
    k = known()["chain"]
    m = W.chain(k["n"], lambda c: 0.0 if c == k["singular_dof"] else 1.0, lambda r, c: 0.0)
    h, err, _ = ffi.factor_indef(m)
    assert h is None and err == k["singular_dof"]


def test_dual_4x4(gpu):
    """src/steps/nlgeom_solver.rs:145-175 through the C interface."""
    k = known()["dual4"]
    a = np.array(k["a"])
    n = 4
    indptr, indices, data = [0], [], []
    for c in range(n):
        for r in range(n):
            if a[r, c] != 0.0:
                indices.append(r)
                data.append(a[r, c])
        indptr.append(len(indices))
    coords = np.zeros(3 * n)
    coords[0::3] = np.arange(n)
    m = W.Model("dual4", n, n, np.arange(n), coords, np.array(indptr), np.array(indices), np.array(data), np.zeros(n),
                None, "full")
    h, err, ine = ffi.factor_indef(m)
    assert h is not None
    assert ine[0] == k["negative"]
    hp, errp, _ = ffi.factor(m)
    assert hp is None  # the positive definite path fails
    x = h.solve(a @ np.array(k["x"]))
    assert np.max(np.abs(x - np.array(k["x"]))) < k["tol"]


@pytest.mark.parametrize("case", [0, 1, 2])
def test_laplace_matches_oracle(gpu, case):
    k = known()["laplace"][case]
    m, below = W.laplace3d(k["g"], k["sigma"])
    h, err, ine = ffi.factor_indef(m)
    ho, erro, ineo = refcpu.factor_indef(m)
    assert h is not None and ho is not None
    assert ine == ineo == (below, 0, m.n - below)
    assert h.info() == ho.info()
    b = np.random.default_rng(2).standard_normal((3, m.n))
    x = h.solve(b)
    xo = ho.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10


def test_shifted_elasticity_matches_oracle(gpu):
    """A C3D8 cube shifted into the indefinite range: 3-DOF nodes, 2×2 pivots and delays."""
    m = W.hex8_cube(5).full()
    d = m.data.copy()
    diag_pos = [m.indptr[c] + int(np.where(m.indices[m.indptr[c]:m.indptr[c + 1]] == c)[0][0]) for c in range(m.n)]
    shift = 0.2 * float(np.median(d[diag_pos]))
    d[diag_pos] -= shift
    ms = W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, d, m.rhs, None, "full")
    h, err, ine = ffi.factor_indef(ms)
    ho, erro, ineo = refcpu.factor_indef(ms)
    assert h is not None and ho is not None
    assert ine == ineo and ine[0] > 0
    x = h.solve(m.rhs)
    xo = ho.solve(m.rhs)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9


def _shifted_cube(n, frac=0.2):
    m = W.hex8_cube(n).full()
    d = m.data.copy()
    diag_pos = [m.indptr[c] + int(np.where(m.indices[m.indptr[c]:m.indptr[c + 1]] == c)[0][0]) for c in range(m.n)]
    d[diag_pos] -= frac * float(np.median(d[diag_pos]))
    return W.Model(m.name + " shifted", m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, d, m.rhs, None, "full")


@pytest.mark.parametrize("n,cluster_rows", [(12, None), (12, "64"), (16, None)])
def test_shifted_cube_matches_oracle(gpu, monkeypatch, n, cluster_rows):
    """C3D8 cubes shifted into the indefinite range (12³: n = 6,084, top fronts of ~1,400
    rows; 16³: n = 13,872): the block rounds with the multi-CTA trailing update give the
    oracle's inertia and solution — with the block rounds of fronts of 768 rows and more on
    clusters of CTAs, and with every front of 64 rows and more on clusters
    (RFG_INDEF_CLUSTER_ROWS=64)."""
    if cluster_rows:
        monkeypatch.setenv("RFG_INDEF_CLUSTER_ROWS", cluster_rows)
    ms = _shifted_cube(n)
    h, err, ine = ffi.factor_indef(ms)
    ho, erro, ineo = refcpu.factor_indef(ms)
    assert h is not None and ho is not None, (err, erro)
    assert ine == ineo and ine[0] > 0
    x = h.solve(ms.rhs)
    xo = ho.solve(ms.rhs)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9


@pytest.mark.parametrize("cluster_rows", [None, "64"])
def test_laplace_20_matches_oracle(gpu, monkeypatch, cluster_rows):
    """The shifted 7-point Laplacian on 20³ nodes (examples/solver_bench.rs:87-157): the
    inertia equals the analytic count and the oracle's, the solution the oracle's (also with
    every front of 64 rows and more on clusters of CTAs)."""
    if cluster_rows:
        monkeypatch.setenv("RFG_INDEF_CLUSTER_ROWS", cluster_rows)
    g = 20
    m, below = W.laplace3d(g, W.laplace_sigma(g))
    h, err, ine = ffi.factor_indef(m)
    ho, erro, ineo = refcpu.factor_indef(m)
    assert h is not None and ho is not None
    assert ine == ineo == (below, 0, m.n - below)
    b = np.random.default_rng(5).standard_normal((2, m.n))
    x = h.solve(b)
    xo = ho.solve(b)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10
