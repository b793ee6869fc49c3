"""GPU parity: the CUDA numeric phase through the C interface against the oracle.

Tolerance: the plain FP64 GPU path must reproduce the oracle's FP64 solution to
a relative error of at most 1e-10 (2-norm) and its pivots D to 1e-10 (max
relative); the mixed path must reach a normwise backward error of 1e-12 after
FP64 refinement. Symbolic data (front list, order, info) must be identical.
"""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, solver, workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def check_pd(model, nrhs=1, seed=0):
    m = model.full()
    h, err, d = ffi.factor(m, want_d=True)
    assert h is not None, f"GPU factor failed at {err}: {ffi.last_error()}"
    ho, erro, do = refcpu.factor(m, want_d=True)
    assert ho is not None
    assert np.array_equal(h.fronts(), ho.fronts())
    assert np.array_equal(h.order(), ho.order())
    assert h.info() == ho.info()
    assert float(np.max(np.abs(d - do) / np.maximum(np.abs(do), 1e-300))) <= TOL
    rng = np.random.default_rng(seed)
    b = m.rhs if nrhs == 1 else rng.standard_normal((nrhs, m.n))
    x = h.solve(b)
    xo = ho.solve(b)
    assert rel(x, xo) <= TOL
    return h, ho


def test_cube_small(gpu):
    check_pd(W.hex8_cube(4))


def test_cube_20_c1(gpu):
    """The 20³ C3D8 cube of the first benchmark configuration (n = 26,460)."""
    h, ho = check_pd(W.hex8_cube(20))
    assert h.fronts().shape[0] == 614


def test_cube_multi_rhs(gpu):
    check_pd(W.hex8_cube(8), nrhs=8)
    check_pd(W.hex8_cube(6), nrhs=40)  # more right-hand sides than one sweep holds


def test_cube_block_rhs_wide_steps(gpu):
    """5 to 32 right-hand sides through the register-tiled sweep kernels, on a cube whose
    top fronts span several 256-pivot solve steps."""
    for nrhs in (5, 16, 32):
        check_pd(W.hex8_cube(12), nrhs=nrhs, seed=nrhs)


def test_mixed_block_rhs_refined(gpu):
    m = W.hex8_cube(12).full()
    h, err, _ = ffi.factor(m, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    ho, _, _ = refcpu.factor(m)
    rng = np.random.default_rng(3)
    for nrhs in (6, 32):
        b = rng.standard_normal((nrhs, m.n))
        x, st = h.solve(b, stats=True)
        assert st["backward_error"] <= 1e-12, st
        assert rel(x, ho.solve(b)) <= 1e-8


def test_plates(gpu):
    for nx, ny in [(20, 2), (57, 5), (200, 20)]:
        check_pd(W.plate(nx, ny), nrhs=3)


def test_hex20(gpu):
    check_pd(W.hex20_cube(3))


def test_ill_conditioned_moduli(gpu):
    n = 8
    check_pd(W.hex8_cube(n, emod=W.log_uniform_moduli(n, seed=0)))


def test_chain_pd_and_refusal(gpu):
    """ffi/src/lib.rs:429-441: tridiag(-1, 2, -1) is PD; shifted by 1.3 the PD path refuses."""
    n = 40
    m = W.chain(n, lambda c: 2.0, lambda r, c: -1.0)
    check_pd(m)
    ms = W.chain(n, lambda c: 2.0 - 1.3, lambda r, c: -1.0)
    h, err, _ = ffi.factor(ms)
    ho, erro, _ = refcpu.factor(ms)
    assert h is None and ho is None
    assert err == erro


def test_not_positive_definite_dof_matches(gpu):
    m = W.hex8_cube(5).full()
    data = m.data.copy()
    # make one interior diagonal entry negative
    c = m.n // 2
    p = np.where((m.indices[m.indptr[c]:m.indptr[c + 1]]) == c)[0][0] + m.indptr[c]
    data[p] = -abs(data[p])
    bad = W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, data, m.rhs, m.graph, "full")
    h, err, _ = ffi.factor(bad)
    ho, erro, _ = refcpu.factor(bad)
    assert h is None and ho is None
    assert err == erro and err >= 0


def test_uncoupled_dofs(gpu):
    """Diagonal-only DOFs are split off and solved by division (ffi/src/lib.rs:105-128, 353-355)."""
    base = W.hex8_cube(3).full()
    n0 = base.n
    extra = 5
    n = n0 + extra
    indptr = np.concatenate([base.indptr, base.indptr[-1] + np.arange(1, extra + 1)])
    indices = np.concatenate([base.indices, np.arange(n0, n)])
    data = np.concatenate([base.data, np.linspace(1.0, 5.0, extra)])
    loc = np.concatenate([base.loc, np.full(extra, 0)])
    m = W.Model("cube+iso", n, base.nn, loc, base.coords, indptr, indices, data, np.ones(n), None, "full")
    h, err, d = ffi.factor(m, want_d=True)
    ho, erro, do = refcpu.factor(m, want_d=True)
    assert h is not None and ho is not None
    assert np.array_equal(h.order(), ho.order())
    assert rel(d, do) <= TOL
    b = np.random.default_rng(1).standard_normal((2, n))
    assert rel(h.solve(b), ho.solve(b)) <= TOL
    # an uncoupled DOF with a non-positive diagonal is refused with its DOF
    data2 = data.copy()
    data2[-2] = 0.0
    m2 = W.Model("cube+iso0", n, base.nn, loc, base.coords, indptr, indices, data2, np.ones(n), None, "full")
    h2, err2, _ = ffi.factor(m2)
    ho2, erro2, _ = refcpu.factor(m2)
    assert h2 is None and ho2 is None and err2 == erro2 == n - 2


def test_empty_system(gpu):
    m = W.Model("empty", 0, 0, np.zeros(0, np.int64), np.zeros(0), np.zeros(1, np.int64), np.zeros(0, np.int64),
                np.zeros(0), np.zeros(0), None, "full")
    h, err, _ = ffi.factor(m)
    assert h is not None
    assert h.info() == (0.0, 0)
    x = h.solve(np.zeros(0))
    assert x.size == 0


def test_invalid_input(gpu):
    m = W.hex8_cube(2).full()
    bad = W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices.copy(), m.data, m.rhs, None, "full")
    bad.indices[3] = m.n + 7
    h, err, _ = ffi.factor(bad)
    assert h is None and err == -1


def test_refactor_same_pattern(gpu):
    m = W.hex8_cube(6).full()
    h, err, _ = ffi.factor(m)
    m2 = W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, m.data * 3.0, m.rhs, None, "full")
    assert h.refactor(m2.data) == -1
    ho, _, _ = refcpu.factor(m2)
    assert rel(h.solve(m.rhs), ho.solve(m.rhs)) <= TOL


def test_engine_api_matches_oracle(gpu):
    """LinearSolver::prepare → add → factor → solve (src/solver/api.rs) with leaf 48."""
    m = W.hex8_cube(7)
    sm = solver.select("direct-gpu").prepare(m.graph)
    sym = refcpu.Symbolic(m.graph, 48)
    assert np.array_equal(sm.first_dof(), sym.first_dof())
    colptr, rowidx, val, eq = refcpu.to_internal(m, sym)
    cols = np.repeat(np.arange(sm.n()), np.diff(colptr))
    sm.zero()
    sm.add_many(rowidx, cols, val)
    sm.factor()
    b = np.zeros(sm.n())
    b[eq] = m.rhs
    x = b.copy()
    sm.solve(x)
    F, e = sym.pd_factor(colptr, rowidx, val)
    assert e == -1
    assert rel(x, F.solve(b)) <= TOL


def test_engine_api_not_pd(gpu):
    m = W.hex8_cube(3)
    sm = solver.select().prepare(m.graph)
    sym = refcpu.Symbolic(m.graph, 48)
    colptr, rowidx, val, eq = refcpu.to_internal(m, sym)
    val = val.copy()
    val[colptr[10]] = -1.0  # diagonal of equation 10
    cols = np.repeat(np.arange(sm.n()), np.diff(colptr))
    sm.add_many(rowidx, cols, val)
    with pytest.raises(solver.NotPositiveDefinite) as ei:
        sm.factor()
    F, e = sym.pd_factor(colptr, rowidx, val)
    assert F is None and ei.value.eq == e


@pytest.mark.parametrize("emod", [None, "log"])
def test_mixed_precision_refined(gpu, emod):
    n = 10
    model = W.hex8_cube(n, emod=W.log_uniform_moduli(n, seed=0) if emod else None).full()
    h, err, _ = ffi.factor(model, precision=ffi.MIXED, tensor_cores=False)
    assert h is not None, ffi.last_error()
    x, st = h.solve(model.rhs, stats=True)
    ho, _, _ = refcpu.factor(model)
    xo = ho.solve(model.rhs)
    assert st["backward_error"] <= 1e-12, st
    assert rel(x, xo) <= 1e-8, (rel(x, xo), st)


def test_fp64_reports_backward_error(gpu):
    m = W.hex8_cube(8).full()
    h, err, _ = ffi.factor(m)
    x, st = h.solve(m.rhs, stats=True)
    assert st["iterations"] == 0
    assert st["backward_error"] <= 1e-13



def test_device_entry_points_wait_for_the_callers_stream(gpu):
    """rfg_refactor_device / rfg_solve_device read inputs that the caller wrote on the
    legacy default stream (torch's default stream) without a synchronize: the handle's
    stream waits for that work on entry."""
    import torch

    m = W.hex8_cube(10).full()
    h, err, _ = ffi.factor(m)
    assert h is not None, ffi.last_error()
    ho, _, _ = refcpu.factor(m)
    xo = ho.solve(m.rhs)
    data_d = torch.zeros(len(m.data), dtype=torch.float64, device="cuda")
    b_d = torch.zeros(m.n, dtype=torch.float64, device="cuda")
    busy = torch.randn(4096, 4096, dtype=torch.float64, device="cuda")
    for trial in range(3):
        torch.cuda.synchronize()
        data_d.zero_()
        b_d.zero_()
        for _ in range(4):  # tens of milliseconds of work ahead of the copies
            busy = busy @ busy
            busy = busy / busy.abs().max()
        data_d.copy_(torch.from_numpy(m.data).to("cuda", non_blocking=False) + 0.0 * busy[0, 0])
        b_d.copy_(torch.from_numpy(m.rhs).cuda() + 0.0 * busy[0, 1])
        assert h.refactor_device(data_d.data_ptr()) == -1, ffi.last_error()
        h.solve_device(b_d.data_ptr(), 1)
        torch.cuda.synchronize()
        assert rel(b_d.cpu().numpy(), xo) <= TOL, trial
    h.free()


def test_pivot_reciprocal_within_one_ulp(gpu):
    """The pivot blocks divide by each pivot through a Newton–Raphson reciprocal instead of
    the IEEE division: within one unit in the last place of the correctly rounded 1/x over
    twenty decades and at the ends of the mantissa."""
    import ctypes

    rng = np.random.default_rng(11)
    x = np.concatenate([10.0 ** rng.uniform(-10, 10, 200000), [1.0, 2.0, 0.5, np.nextafter(1.0, 2.0),
                                                               np.nextafter(2.0, 1.0), 3.0, 1e-300, 1e300]])
    r = np.zeros_like(x)
    f64 = ctypes.POINTER(ctypes.c_double)
    assert ffi.lib().rfg_selftest_reciprocal(x.ctypes.data_as(f64), r.ctypes.data_as(f64), x.size) == 0
    exact = 1.0 / x
    ulp = np.abs(r - exact) / np.spacing(exact)
    assert ulp.max() <= 1.0, float(ulp.max())
