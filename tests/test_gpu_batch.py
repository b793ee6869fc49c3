"""Batched factorization of many independent models (rfg_batch_factor) against
the oracle, model by model: FP64 to 1e-10, mixed after refinement to a backward
error of 1e-12."""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def plates(count, seed=3):
    return [W.plate(nx, ny).full().with_rhs(8, seed=100 + i) for i, (nx, ny) in
            enumerate(W.plate_sizes(count, seed=seed))]


def test_batch_plates_fp64(gpu):
    models = plates(24)
    bh, em, ed = ffi.factor_batch(models)
    assert bh is not None, (em, ed, ffi.last_error())
    xs = bh.solve_models([m.rhs for m in models])
    for m, x in zip(models, xs):
        ho, _, _ = refcpu.factor(m)
        assert rel(x, ho.solve(m.rhs)) <= 1e-10


def test_batch_mixed_refined(gpu):
    models = plates(12, seed=5) + [W.hex8_cube(6).full().with_rhs(8, seed=9)]
    bh, em, ed = ffi.factor_batch(models, precision=ffi.MIXED)
    assert bh is not None, ffi.last_error()
    xs, st = bh.solve_models([m.rhs for m in models], stats=True)
    assert st["backward_error"] <= 1e-12, st
    for m, x in zip(models, xs):
        ho, _, _ = refcpu.factor(m)
        # slender cantilever plates are badly conditioned: forward error ≈ κ·(backward error)
        assert rel(x, ho.solve(m.rhs)) <= 1e-5


def test_batch_refactor_and_error_model(gpu):
    models = plates(6, seed=7)
    bh, em, ed = ffi.factor_batch(models)
    assert bh is not None
    # new values: every model scaled differently
    scaled = [W.Model(m.name, m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, m.data * (i + 2), m.rhs, None, "full")
              for i, m in enumerate(models)]
    assert bh.refactor(np.concatenate([m.data for m in scaled])) == -1
    xs = bh.solve_models([m.rhs for m in scaled])
    for m, x in zip(scaled, xs):
        ho, _, _ = refcpu.factor(m)
        assert rel(x, ho.solve(m.rhs)) <= 1e-10
    # a model that is not positive definite is reported with its index and DOF
    bad = models[3]
    data = bad.data.copy()
    c = bad.n // 2
    p = bad.indptr[c] + int(np.where(bad.indices[bad.indptr[c]:bad.indptr[c + 1]] == c)[0][0])
    data[p] = -data[p]
    badm = W.Model(bad.name, bad.n, bad.nn, bad.loc, bad.coords, bad.indptr, bad.indices, data, bad.rhs, None, "full")
    bh2, em2, ed2 = ffi.factor_batch(models[:3] + [badm] + models[4:])
    ho, erro, _ = refcpu.factor(badm)
    assert bh2 is None and em2 == 3 and ed2 == erro
