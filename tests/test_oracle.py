"""The oracle (CPU restatement of the reference) pinned against the reference's
own known answers and the golden fixtures of tests/golden/."""
import json
import os

import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def known():
    with open(os.path.join(GOLD, "known_answers.json")) as f:
        return json.load(f)


def test_chain_inertia_and_refusal():
    """ffi/src/lib.rs:429-456."""
    k = known()["chain"]
    n, sigma = k["n"], k["sigma"]
    m = W.chain(n, lambda c: 2.0 - sigma, lambda r, c: -1.0)
    h, err, _ = refcpu.factor(m)
    assert h is None  # the positive definite path must refuse
    h, err, ine = refcpu.factor_indef(m)
    assert h is not None
    assert list(ine) == k["inertia"]
    assert h.inertia() == tuple(k["inertia"])
    b = np.sin(np.arange(n) * 0.3)
    x = h.solve(b)
    assert np.max(np.abs(m.dense() @ x - b)) < k["residual_tol"]


def test_chain_singular_dof():
    """ffi/src/lib.rs:472-476: a zero DOF 7 gives err_dof = 7."""
    k = known()["chain"]
    m = W.chain(k["n"], lambda c: 0.0 if c == k["singular_dof"] else 1.0, lambda r, c: 0.0)
    h, err, _ = refcpu.factor_indef(m)
    assert h is None and err == k["singular_dof"]


def test_dual_indefinite_4x4():
    """src/steps/nlgeom_solver.rs:145-175: direct fails, indefinite gives 2 negative
    eigenvalues and the exact solution."""
    k = known()["dual4"]
    a = np.array(k["a"])
    g = W.Graph(np.array([[i, 0.0, 0.0] for i in range(4)]), np.array([0, 1, 3, 5, 6]), np.array([1, 0, 2, 1, 3, 2]),
                np.ones(4, np.int64))
    sym = refcpu.Symbolic(g, 48)
    fd = sym.first_dof()
    colptr, rowidx = sym.pattern()
    val = np.zeros(len(rowidx))
    for i in range(4):
        for j in range(i + 1):
            if a[i, j] != 0.0:
                r, c = max(fd[i], fd[j]), min(fd[i], fd[j])
                p = colptr[c] + np.searchsorted(rowidx[colptr[c]:colptr[c + 1]], r)
                val[p] += a[i, j]
    F, e = sym.pd_factor(colptr, rowidx, val)
    assert F is None and e >= 0
    F, e = sym.indef_factor(colptr, rowidx, val)
    assert F is not None and F.stats()["neg"] == k["negative"]
    x = np.array(k["x"])
    b = np.zeros(4)
    b[fd] = a @ x
    y = F.solve(b)
    assert np.max(np.abs(y[fd] - x)) < k["tol"]


@pytest.mark.parametrize("case", [0, 1, 2])
def test_laplace_inertia_is_analytic(case):
    """examples/solver_bench.rs:87-157: the number of negative pivots equals the
    analytic count of eigenvalues below σ."""
    k = known()["laplace"][case]
    m, below = W.laplace3d(k["g"], k["sigma"])
    assert below == k["below"]
    h, err, ine = refcpu.factor_indef(m)
    assert h is not None
    assert ine[0] == k["below"] and ine[1] == 0 and ine[2] == m.n - k["below"]
    b = np.random.default_rng(0).standard_normal(m.n)
    x = h.solve(b)
    assert np.linalg.norm(m.matvec(x) - b) / np.linalg.norm(b) < 1e-10


def test_pd_solution_matches_dense():
    m = W.hex8_cube(3).full()
    h, err, d = refcpu.factor(m, want_d=True)
    x = h.solve(m.rhs)
    xd = np.linalg.solve(m.dense(), m.rhs)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-12
    # pivots D are positive and their product's logarithm matches the determinant
    sign, logdet = np.linalg.slogdet(m.dense())
    assert sign > 0 and abs(np.sum(np.log(d)) - logdet) < 1e-8 * abs(logdet)


def test_pd_ffi_keeps_reference_lower_only_semantics():
    """The reference's positive definite C path keeps only entries with internal row >=
    internal column (ffi/src/lib.rs:216-224), so a lower-only CSC is not the same matrix."""
    m = W.hex8_cube(3)
    h_low, _, _ = refcpu.factor(m)
    h_full, _, _ = refcpu.factor(m.full())
    xl = h_low.solve(m.rhs)
    xf = h_full.solve(m.rhs)
    assert np.linalg.norm(xl - xf) / np.linalg.norm(xf) > 1e-6


def test_cube20_front_statistics():
    k = known()["cube20"]
    m = W.hex8_cube(20)
    assert m.n == k["n"]
    s48 = refcpu.Symbolic(m.graph, 48)
    s16 = refcpu.Symbolic(m.graph, 16)
    assert s48.nfronts == k["fronts_leaf48"] and s16.nfronts == k["fronts_leaf16"]
    assert abs(s48.work() / k["work_leaf48"] - 1) < 1e-3
    assert abs(s48.factor_size() / k["factor_size_leaf48"] - 1) < 1e-2
    f = s48.fronts()
    big = f[np.argmax(f[:, 1] + f[:, 2])]
    assert [int(big[1]), int(big[2])] == k["largest_front"]


@pytest.mark.parametrize("name", ["hex8_6", "plate_40x4", "hex20_2"])
@pytest.mark.parametrize("leaf", [48, 16])
def test_symbolic_matches_golden(name, leaf):
    with open(os.path.join(GOLD, f"symbolic_{name}_leaf{leaf}.json")) as f:
        g = json.load(f)
    mesh = {"hex8_6": lambda: W.hex8_cube(6), "plate_40x4": lambda: W.plate(40, 4),
            "hex20_2": lambda: W.hex20_cube(2)}[name]()
    s = refcpu.Symbolic(mesh.graph, leaf)
    assert s.n == g["n"]
    assert s.fronts().tolist() == g["fronts"]
    assert s.first_dof().tolist() == g["first_dof"]
    assert s.rows().tolist() == g["rows"]
    assert s.children().tolist() == g["children"]
    assert s.work() == g["work"]
    assert s.factor_size() == g["factor_size"]


def test_threads_do_not_change_results():
    m = W.hex8_cube(12).full()
    refcpu.set_threads(1)
    h1, _, d1 = refcpu.factor(m, want_d=True)
    x1 = h1.solve(m.rhs)
    refcpu.set_threads(8)
    h8, _, d8 = refcpu.factor(m, want_d=True)
    x8 = h8.solve(m.rhs)
    refcpu.set_threads(0)
    assert np.array_equal(d1, d8) and np.array_equal(x1, x8)


@pytest.mark.parametrize("nparts", [1, 2, 5, 12])
@pytest.mark.parametrize("case", ["hex8_12", "plate_120x12"])
def test_staged_factor_is_the_plain_factor(case, nparts):
    """oref_staged_* (the reference arm's time slices) gives the factor bit for bit."""
    m = (W.hex8_cube(12) if case == "hex8_12" else W.plate(120, 12)).full()
    h, _, _ = refcpu.factor(m)
    x = h.solve(m.rhs)
    S = refcpu.StagedFactor(m, nparts)
    assert S.nparts == nparts
    assert abs(sum(S.part_work(p) for p in range(nparts)) - h.info()[0]) <= 1e-9 * h.info()[0]
    for p in range(nparts):
        assert S.part(p)
    hs, err = S.finish()
    assert err == -1
    assert np.array_equal(hs.solve(m.rhs), x)
    assert np.array_equal(hs.fronts(), h.fronts()) and np.array_equal(hs.order(), h.order())


def test_staged_factor_reports_the_failing_dof():
    m = W.hex8_cube(8).full()
    m.data = m.data.copy()
    m.data[m.indptr[57]:m.indptr[58]][m.indices[m.indptr[57]:m.indptr[58]] == 57] *= -1.0
    h, err, _ = refcpu.factor(m)
    assert h is None and err >= 0
    S = refcpu.StagedFactor(m, 3)
    oks = [S.part(p) for p in range(3)]
    assert not all(oks)
    hs, err_s = S.finish()
    assert hs is None and err_s == err
