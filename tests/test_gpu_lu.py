"""The GPU multifrontal LU (rustyfem_factor_unsym) against the reference's known answer and
the oracle: the same delayed pivots, the same factor size, the solution to 1e-10."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")


def csc(m):
    return sp.csc_matrix((m.data, m.indices, m.indptr), shape=(m.n, m.n))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_lu_chain_known_answer(gpu):
    """ffi/src/lib.rs:458-469: residual below 1e-10 per row, no inertia for an LU handle."""
    k = json.load(open(GOLD))["lu_chain"]
    n = k["n"]
    m = W.chain(n, lambda c: k["diag"], lambda r, c: k["sub"] if r > c else k["sup"])
    h, err, st = ffi.factor_unsym(m)
    assert h is not None, ffi.last_error()
    b0 = np.sin(np.arange(n) * 0.3)
    x = h.solve(b0)
    assert np.max(np.abs(m.dense() @ x - b0)) < k["residual_tol"]
    assert h.inertia() is None


def test_lu_singular_dof(gpu):
    k = json.load(open(GOLD))["chain"]
    m = W.chain(k["n"], lambda c: 0.0 if c == k["singular_dof"] else 1.0, lambda r, c: 0.0)
    h, err, _ = ffi.factor_unsym(m)
    assert h is None and err == k["singular_dof"]


def test_lu_root_partial_pivoting_matches_the_oracle(gpu):
    """A zero diagonal: every variable is delayed to the root, which pivots by rows."""
    n = 40
    m = W.chain(n, lambda c: 0.0, lambda r, c: -1.3 if r > c else -0.7)
    h, err, st = ffi.factor_unsym(m)
    ho, erro, dlo = refcpu.factor_unsym(m)
    assert h is not None and ho is not None, ffi.last_error()
    assert st["delayed"] == dlo > 0
    assert h.info() == ho.info()
    b = np.cos(np.arange(n) * 0.7)
    assert rel(h.solve(b), ho.solve(b)) < 1e-10


@pytest.mark.parametrize("n,alpha,cluster_rows", [(8, 30.0, None), (12, 30.0, None), (12, 30.0, "64"),
                                                  (16, 30.0, None), (24, 30.0, None)])
def test_lu_delayed_pivots_match_the_oracle(gpu, monkeypatch, n, alpha, cluster_rows):
    """A strong skew-symmetric part makes diagonals fail the threshold test: the GPU takes the
    oracle's pivot decisions (the same delays and factor size) and its solution — with the
    block rounds of fronts of 768 rows and more on clusters of CTAs (16³, 24³), and with every
    front of 64 rows and more on clusters (12³ with RFG_LU_CLUSTER_ROWS=64)."""
    if cluster_rows:
        monkeypatch.setenv("RFG_LU_CLUSTER_ROWS", cluster_rows)
    m = W.skew_perturbed(W.hex8_cube(n), alpha, seed=0)
    h, err, st = ffi.factor_unsym(m)
    ho, erro, dlo = refcpu.factor_unsym(m)
    assert h is not None and ho is not None, (err, erro, ffi.last_error())
    assert st["delayed"] == dlo
    assert h.info() == ho.info()
    b = np.random.default_rng(1).standard_normal((3, m.n))
    x = h.solve(b)
    assert rel(x, ho.solve(b)) < 1e-10
    A = csc(m)
    for j in range(3):
        assert np.linalg.norm(A @ x[j] - b[j]) / np.linalg.norm(b[j]) < 1e-9


def test_lu_unsymmetric_cube_matches_the_oracle(gpu):
    """An unsymmetric perturbation of the 10³ cube's off-diagonal entries (same pattern)."""
    m = W.hex8_cube(10).full()
    d = m.data.copy()
    cols = np.repeat(np.arange(m.n), np.diff(m.indptr))
    off = m.indices != cols
    d[off] *= 1.0 + 0.3 * np.random.default_rng(0).standard_normal(int(off.sum()))
    mu = W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, d, m.rhs, None, "full")
    h, err, st = ffi.factor_unsym(mu)
    ho, _, dlo = refcpu.factor_unsym(mu)
    assert h is not None, ffi.last_error()
    assert st["delayed"] == dlo
    assert np.array_equal(h.order(), ho.order())
    assert rel(h.solve(mu.rhs), ho.solve(mu.rhs)) < 1e-10


def test_lu_of_an_spd_matrix_matches_the_ldlt_path(gpu):
    m = W.hex8_cube(8).full()
    h, err, st = ffi.factor_unsym(m)
    hp, _, _ = ffi.factor(m)
    assert h is not None and st["delayed"] == 0
    assert rel(h.solve(m.rhs), hp.solve(m.rhs)) < 1e-10
