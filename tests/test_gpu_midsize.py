"""Mid-size parity: the 30³ C3D8 cube (n = 86,490, top fronts of several thousand rows)
through both GPU paths against the oracle. At this size the outer Schur updates of the
top fronts run on the large tiles (128×256 tcgen05 tiles in the mixed path, 128-row
FP64 tensor-core tiles in the FP64 path) and the deep pipelines of those kernels are
checked directly, not only through the backward error.

Tolerances: FP64 path, relative error of x ≤ 1e-10 (2-norm) and of the pivots D ≤ 1e-10
(max relative) against the oracle; mixed path, backward error ≤ 1e-12 after refinement,
relative error of x ≤ 1e-8 (homogeneous) / ≤ 1e-6 (E log-uniform over six decades, a
far worse conditioned matrix), pivots D ≤ 1e-4 on the homogeneous cube (the mixed
factor keeps D in FP64 but its fronts in FP32)."""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu

N = 30


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def drel(d, do):
    return float(np.max(np.abs(d - do) / np.abs(do)))


@pytest.fixture(scope="module", params=["steel", "log_uniform"])
def case(request):
    emod = W.log_uniform_moduli(N, seed=0) if request.param == "log_uniform" else None
    m = W.hex8_cube(N, emod=emod).full()
    ho, err, do = refcpu.factor(m, want_d=True)
    assert ho is not None, err
    xo = ho.solve(m.rhs)
    fronts, order, info = ho.fronts(), ho.order(), ho.info()
    ho.free()
    return request.param, m, xo, do, fronts, order, info


def test_uses_the_large_tiles(gpu, case):
    _, m, *_ = case
    sym = ffi.Symbolic(m.graph, 16)
    fl = sym.plan_flops()
    assert fl["outer_128tiles"] > 0.5 * fl["outer"] and fl["tiles_128"] > 0, fl


def test_fp64_matches_oracle(gpu, case):
    name, m, xo, do, fronts, order, info = case
    h, err, d = ffi.factor(m, want_d=True)
    assert h is not None, ffi.last_error()
    assert np.array_equal(h.fronts(), fronts) and np.array_equal(h.order(), order) and h.info() == info
    assert drel(d, do) <= 1e-10
    x = h.solve(m.rhs)
    assert rel(x, xo) <= 1e-10, (name, rel(x, xo))
    h.free()


def test_mixed_matches_oracle(gpu, case):
    name, m, xo, do, *_ = case
    h, err, d = ffi.factor(m, precision=ffi.MIXED, want_d=True)
    assert h is not None, ffi.last_error()
    x, st = h.solve(m.rhs, stats=True)
    assert st["backward_error"] <= 1e-12, st
    assert rel(x, xo) <= (1e-6 if name == "log_uniform" else 1e-8), (name, rel(x, xo), st)
    if name == "steel":
        assert drel(d, do) <= 1e-4, drel(d, do)
    h.free()
