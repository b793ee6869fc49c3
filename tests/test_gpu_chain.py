"""Solve chains: the sweeps of the levels with few fronts run as one launch per level and
direction (clusters of four CTAs per 256-pivot diagonal block, bounded waits on the blocks
they depend on) instead of two launches per 256-pivot step.

* One sweep of the same FP32 factor with and without chains: the two solutions differ only
  by the rounding of the sweep (the chain multiplies by the inverse of each 256 × 256
  diagonal block instead of substituting block by block), far below the factor's own error.
* RFG_SOLVE_CHAIN = 100000 puts every level on chains: many small fronts, blocks narrower
  than 256 pivots, CTAs of a cluster without rows or columns, the later rows of every front.
* Refined solutions against the oracle, with 1 to 4 right-hand sides (the kernels'
  right-hand-side widths).
"""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _solve(model, b, refine):
    h, err, _ = ffi.factor(model, precision=ffi.MIXED, refine_max_iter=-1 if refine else 0)
    assert h is not None, ffi.last_error()
    try:
        return h.solve(b, stats=True)
    finally:
        h.free()


@pytest.mark.parametrize("n", [12, 20])
@pytest.mark.parametrize("chain", ["8", "100000"])
def test_chain_sweep_matches_stepped_sweep(gpu, monkeypatch, n, chain):
    model = W.hex8_cube(n).full()
    rng = np.random.default_rng(n)
    for nrhs in (1, 2, 3, 4):
        b = model.rhs if nrhs == 1 else rng.standard_normal((nrhs, model.n))
        monkeypatch.setenv("RFG_SOLVE_CHAIN", "0")
        x0, st0 = _solve(model, b, refine=False)
        monkeypatch.setenv("RFG_SOLVE_CHAIN", chain)
        x1, st1 = _solve(model, b, refine=False)
        assert st1["launches"] != st0["launches"], (st0, st1)  # the chain launches ran
        assert rel(x1, x0) <= 1e-10, (nrhs, rel(x1, x0))


@pytest.mark.parametrize("chain", ["8", "100000"])
def test_chain_refined_against_oracle(gpu, monkeypatch, chain):
    model = W.hex8_cube(16).full()
    ho, _, _ = refcpu.factor(model)
    rng = np.random.default_rng(3)
    monkeypatch.setenv("RFG_SOLVE_CHAIN", chain)
    for nrhs in (1, 3):
        b = model.rhs if nrhs == 1 else rng.standard_normal((nrhs, model.n))
        x, st = _solve(model, b, refine=True)
        xo = np.stack([ho.solve(bb) for bb in np.atleast_2d(b)]).reshape(np.shape(b))
        assert st["backward_error"] <= 1e-12, st
        assert rel(x, xo) <= 1e-8, (nrhs, rel(x, xo), st)


def test_chain_plate_and_refactor(gpu, monkeypatch):
    """A 2D model (many small fronts at every level) on chains everywhere, factored twice:
    the chain blocks' inverses must be formed again for the new values. A thin plate in
    bending is far worse conditioned than the cube: the forward error bar follows the
    condition number (as for the log-uniform cubes)."""
    monkeypatch.setenv("RFG_SOLVE_CHAIN", "100000")
    m = W.plate(60, 6).full()
    h, err, _ = ffi.factor(m, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    try:
        ho, _, _ = refcpu.factor(m)
        x, st = h.solve(m.rhs, stats=True)
        assert st["backward_error"] <= 1e-12 and rel(x, ho.solve(m.rhs)) <= 1e-6, st
        m2 = W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, m.data * 3.0, m.rhs, None, "full")
        assert h.refactor(m2.data) == -1
        x2, st2 = h.solve(m.rhs, stats=True)
        assert st2["backward_error"] <= 1e-12, st2
        assert rel(x2, x / 3.0) <= 1e-6
    finally:
        h.free()
