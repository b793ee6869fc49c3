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
    """Mixed path: candidates are (cutover, tensor-core outer tile width) pairs, both
    widths measured; the handle is built with the fastest pair."""
    m = W.hex8_cube(24).full()
    h, err, _ = ffi.factor(m, precision=ffi.MIXED, autotune=True)
    assert h is not None, ffi.last_error()
    rep = h.tune_report_ex()
    assert len(rep) >= 4, rep
    cands = [(c, tn) for c, tn, _ in rep]
    assert len(set(cands)) == len(cands)
    assert {tn for _, tn in cands} == {128, 256}
    best = min(rep, key=lambda r: r[2])
    st0 = h.stats()
    assert (st0["tile_cutover_rows"], st0["outer_tile_n"]) == (best[0], best[1])
    x, st = h.solve(m.rhs, stats=True)
    assert st["backward_error"] <= 1e-12, st
    # the same analysis on the same device is served from the cache
    h2, _, _ = ffi.factor(m, precision=ffi.MIXED, autotune=True)
    assert h2.tune_report_ex() == rep and h2.stats()["tile_cutover_rows"] == best[0]
    h.free()
    h2.free()


@pytest.mark.parametrize("tn", [128, 256])
def test_both_outer_tile_widths_match_the_oracle(gpu, monkeypatch, tn):
    """The tensor-core outer update on 128×128 and on 128×256 tiles (the autotuner's two
    shapes) refines to 1e-12 and matches the oracle."""
    m = W.hex8_cube(20).full()
    ho, _, _ = refcpu.factor(m)
    xo = ho.solve(m.rhs)
    monkeypatch.setenv("RFG_TC_OUTER_TN", str(tn))
    h, err, _ = ffi.factor(m, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    assert h.stats()["outer_tile_n"] == tn
    x, st = h.solve(m.rhs, stats=True)
    assert st["backward_error"] <= 1e-12, st
    assert rel(x, xo) <= 1e-8
    h.free()


def test_fp64_autotune_keeps_parity(gpu):
    m = W.hex8_cube(14).full()
    h, err, _ = ffi.factor(m, precision=ffi.FP64, autotune=True)
    assert h is not None, ffi.last_error()
    assert h.stats()["tile_cutover_rows"] in [c for c, _ in h.tune_report()]
    ho, _, _ = refcpu.factor(m)
    assert rel(h.solve(m.rhs), ho.solve(m.rhs)) <= 1e-10
    h.free()
