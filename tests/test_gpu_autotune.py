"""The cutover autotuner (RFG_FLAG_AUTOTUNE): it measures distinct candidate cutovers,
builds the handle with the fastest one, and the tuned factorization keeps the
accuracy bars (FP64 against the oracle, mixed after refinement)."""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_mixed_autotune_picks_the_fastest_candidate(gpu):
    m = W.hex8_cube(24).full()
    h, err, _ = ffi.factor(m, precision=ffi.MIXED, autotune=True)
    assert h is not None, ffi.last_error()
    rep = h.tune_report()
    assert len(rep) >= 2, rep
    cands = [c for c, _ in rep]
    assert len(set(cands)) == len(cands)
    best = min(rep, key=lambda cm: cm[1])[0]
    assert h.stats()["tile_cutover_rows"] == best
    x, st = h.solve(m.rhs, stats=True)
    assert st["backward_error"] <= 1e-12, st
    # the same analysis on the same device is served from the cache
    h2, _, _ = ffi.factor(m, precision=ffi.MIXED, autotune=True)
    assert h2.tune_report() == rep and h2.stats()["tile_cutover_rows"] == best
    h.free()
    h2.free()


def test_fp64_autotune_keeps_parity(gpu):
    m = W.hex8_cube(14).full()
    h, err, _ = ffi.factor(m, precision=ffi.FP64, autotune=True)
    assert h is not None, ffi.last_error()
    assert h.stats()["tile_cutover_rows"] in [c for c, _ in h.tune_report()]
    ho, _, _ = refcpu.factor(m)
    assert rel(h.solve(m.rhs), ho.solve(m.rhs)) <= 1e-10
    h.free()
