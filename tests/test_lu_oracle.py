"""The oracle's restatement of the unsymmetric multifrontal LU (src/sparse/lu.rs, through
rustyfem_factor_unsym of ffi/src/lib.rs:300-311): the reference's own known answer (the
convection–diffusion chain of ffi/src/lib.rs:458-469), singular input, delayed pivots, the
root's partial pivoting, and agreement with the positive definite path on an SPD matrix."""
import json
import os

import numpy as np
import scipy.sparse as sp

from oracle import refcpu
from rustyfem_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")


def csc(m):
    return sp.csc_matrix((m.data, m.indices, m.indptr), shape=(m.n, m.n))


def test_lu_chain_known_answer():
    k = json.load(open(GOLD))["lu_chain"]
    n = k["n"]
    m = W.chain(n, lambda c: k["diag"], lambda r, c: k["sub"] if r > c else k["sup"])
    h, err, delayed = refcpu.factor_unsym(m)
    assert h is not None and err == -1
    b0 = np.sin(np.arange(n) * 0.3)
    x = h.solve(b0)
    assert np.max(np.abs(m.dense() @ x - b0)) < k["residual_tol"]
    assert h.inertia() is None  # rustyfem_inertia returns -1 for an LU handle


def test_lu_singular_dof():
    k = json.load(open(GOLD))["chain"]
    m = W.chain(k["n"], lambda c: 0.0 if c == k["singular_dof"] else 1.0, lambda r, c: 0.0)
    h, err, _ = refcpu.factor_unsym(m)
    assert h is None and err == k["singular_dof"]


def test_lu_zero_diagonal_delays_to_the_root():
    """A chain with a zero diagonal: no leaf pivot passes the test, everything is delayed to
    the root, which factors it with partial pivoting."""
    n = 40
    m = W.chain(n, lambda c: 0.0, lambda r, c: -1.3 if r > c else -0.7)
    h, err, delayed = refcpu.factor_unsym(m)
    assert h is not None and delayed > 0
    b = np.cos(np.arange(n) * 0.7)
    x = h.solve(b)
    A = m.dense()
    # normwise backward error (the solution grows like (1.3/0.7)^(n/2))
    eta = np.linalg.norm(A @ x - b) / (np.linalg.norm(A, 2) * np.linalg.norm(x) + np.linalg.norm(b))
    assert eta < 1e-15


def test_lu_delays_in_a_3d_front_tree():
    m = W.skew_perturbed(W.hex8_cube(12), 30.0, seed=0)
    h, err, delayed = refcpu.factor_unsym(m)
    assert h is not None and delayed > 100
    x = h.solve(m.rhs)
    assert np.linalg.norm(csc(m) @ x - m.rhs) / np.linalg.norm(m.rhs) < 1e-10


def test_lu_on_an_spd_matrix_matches_the_ldlt_path():
    m = W.hex8_cube(6).full()
    h, err, delayed = refcpu.factor_unsym(m)
    hp, _, _ = refcpu.factor(m)
    assert h is not None and delayed == 0
    x, xp = h.solve(m.rhs), hp.solve(m.rhs)
    assert np.linalg.norm(x - xp) / np.linalg.norm(xp) < 1e-12
