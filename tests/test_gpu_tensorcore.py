"""The mixed-precision path with the tensor-core (tcgen05, 3×TF32) Schur update
against the oracle: after FP64 refinement the backward error must reach 1e-12
and the solution must match the oracle's FP64 solution to 1e-8."""
import numpy as np
import pytest

from oracle import refcpu
from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("n,emod", [(12, None), (16, None), (14, "log")])
def test_mixed_tensor_cores(gpu, n, emod):
    model = W.hex8_cube(n, emod=W.log_uniform_moduli(n, seed=0) if emod else None).full()
    h, err, _ = ffi.factor(model, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    x, st = h.solve(model.rhs, stats=True)
    ho, _, _ = refcpu.factor(model)
    xo = ho.solve(model.rhs)
    assert st["backward_error"] <= 1e-12, st
    # forward error ~ condition number × backward error: E spanning six decades is far
    # worse conditioned than the homogeneous cube
    assert rel(x, xo) <= (1e-6 if emod else 1e-8), (rel(x, xo), st)


def test_tensor_core_factor_matches_simt(gpu):
    """Before refinement, the tensor-core factor solves about as well as the FP32 CUDA-core one."""
    model = W.hex8_cube(16).full()
    sols = []
    for tcores in (False, True):
        h, err, _ = ffi.factor(model, precision=ffi.MIXED, refine_max_iter=0, tensor_cores=tcores)
        assert h is not None, ffi.last_error()
        x, st = h.solve(model.rhs, stats=True)
        sols.append((x, st))
    ho, _, _ = refcpu.factor(model)
    xo = ho.solve(model.rhs)
    e_simt, e_tc = rel(sols[0][0], xo), rel(sols[1][0], xo)
    assert e_tc < 1e-3 and e_tc < 50 * max(e_simt, 1e-7), (e_simt, e_tc)


def test_persistent_kernel_matches_one_tile_per_cta(gpu, monkeypatch):
    """With the TF32 split and one outer block per pass, the persistent warp-specialised
    tensor-core kernel and the one-tile-per-CTA kernel (RFG_TC_PERSISTENT=0) run the same MMA
    sequence per 128×128 tile: their pivots must agree to FP32 rounding and both factors must
    refine to 1e-12."""
    model = W.hex8_cube(18).full()
    out = {}
    monkeypatch.setenv("RFG_TC_KIND", "tf32")
    monkeypatch.setenv("RFG_TC_PAIR", "0")
    for mode in ("0", "1"):
        monkeypatch.setenv("RFG_TC_PERSISTENT", mode)
        h, err, d = ffi.factor(model, precision=ffi.MIXED, want_d=True)
        assert h is not None, ffi.last_error()
        x, st = h.solve(model.rhs, stats=True)
        assert st["backward_error"] <= 1e-12, (mode, st)
        out[mode] = (d, x)
        h.free()
    d0, d1 = out["0"][0], out["1"][0]
    assert float(np.max(np.abs(d0 - d1) / np.abs(d0))) <= 1e-6
    assert rel(out["1"][1], out["0"][1]) <= 1e-9


def test_profiled_graph_replay_times_every_phase(gpu):
    """With profiling on, the numeric phase still replays a CUDA graph; its phase events are
    event-record nodes of that graph, and the phases add up to the factorization time."""
    model = W.hex8_cube(16).full()
    h, err, _ = ffi.factor(model, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    h.set_profiling(True)
    for it in range(3):
        assert h.refactor(model.data) == -1, ffi.last_error()
        st = h.stats()
        ph = st["phase_ms"]
        assert all(p >= 0 for p in ph) and ph[2] > 0 and ph[6] > 0, ph
        # the first replay of a newly captured graph also uploads it; compare the later ones
        if it > 0:
            assert abs(sum(ph) - st["t_factor_ms"]) <= 0.25 * st["t_factor_ms"] + 0.05, (ph, st["t_factor_ms"])
        assert st["schur_launches"] > 0 and st["schur_ms"] == ph[6]
    # level 2: events around the 128-tile outer updates only; the same launches are counted
    # and nothing else is timed
    n1 = st["schur_launches"]
    h.set_profiling(2)
    for it in range(2):
        assert h.refactor(model.data) == -1, ffi.last_error()
        st = h.stats()
        ph = st["phase_ms"]
        assert st["schur_launches"] == n1 and st["schur_ms"] == ph[6] > 0, st
        assert all(p == 0 for p in ph[:6]), ph
        assert st["schur_ms"] < st["t_factor_ms"]
    h.set_profiling(False)
    x, sst = h.solve(model.rhs, stats=True)
    assert sst["backward_error"] <= 1e-12
    h.free()


@pytest.mark.parametrize("n,emod", [(16, None), (14, "log")])
def test_fp16_split_matches_tf32_split(gpu, monkeypatch, n, emod):
    """The FP16 split of U = L·D^(1/2) (default) and the TF32 split of W and L
    (RFG_TC_KIND=tf32) both refine to 1e-12 and reach the same accuracy against the oracle;
    before refinement their factors solve about equally well."""
    model = W.hex8_cube(n, emod=W.log_uniform_moduli(n, seed=0) if emod else None).full()
    ho, _, _ = refcpu.factor(model)
    xo = ho.solve(model.rhs)
    res = {}
    for kind in ("fp16", "tf32"):
        if kind == "tf32":
            monkeypatch.setenv("RFG_TC_KIND", "tf32")
        else:
            monkeypatch.delenv("RFG_TC_KIND", raising=False)
        h, err, _ = ffi.factor(model, precision=ffi.MIXED)
        assert h is not None, ffi.last_error()
        assert h.stats()["tc_kind"] == (2 if kind == "fp16" else 1)
        x, st = h.solve(model.rhs, stats=True)
        assert st["backward_error"] <= 1e-12, (kind, st)
        h0, _, _ = ffi.factor(model, precision=ffi.MIXED, refine_max_iter=0)
        x0 = h0.solve(model.rhs)
        res[kind] = (rel(x, xo), rel(x0, xo), st["iterations"])
        h.free()
        h0.free()
    tol = 1e-6 if emod else 1e-8
    assert res["fp16"][0] <= tol and res["tf32"][0] <= tol, res
    # unrefined: the FP16 split is within a small factor of the TF32 split
    assert res["fp16"][1] <= 10 * max(res["tf32"][1], 1e-9), res


def test_fp16_split_falls_back_to_tf32(gpu, monkeypatch):
    """A row whose scale is not valid (here: every row, through the test switch that
    withholds the original diagonal) makes the engine factor again with the TF32 split."""
    model = W.hex8_cube(14).full()
    monkeypatch.setenv("RFG_TC_H16_FALLBACK_TEST", "1")
    h, err, _ = ffi.factor(model, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    assert h.stats()["tc_kind"] == 1
    x, st = h.solve(model.rhs, stats=True)
    assert st["backward_error"] <= 1e-12, st
    assert h.refactor(model.data) == -1 and h.stats()["tc_kind"] == 1
    h.free()


def test_auto_precision_chooses_per_model(gpu):
    """RFG_AUTO: FP64 for models of small fronts (2D plates, a 12³ cube), mixed precision
    with refinement for the 20³ cube whose large fronts carry most of the flops; either way
    the result meets the bar of the chosen path."""
    for m, want in [(W.plate(200, 20), ffi.FP64), (W.hex8_cube(12), ffi.FP64), (W.hex8_cube(20), ffi.MIXED)]:
        m = m.full()
        h, err, _ = ffi.factor(m, precision=ffi.AUTO)
        assert h is not None, ffi.last_error()
        assert h.stats()["precision"] == want, (m.name, h.stats()["precision"])
        x, st = h.solve(m.rhs, stats=True)
        ho, _, _ = refcpu.factor(m)
        xo = ho.solve(m.rhs)
        if want == ffi.MIXED:
            assert st["backward_error"] <= 1e-12 and st["iterations"] >= 1, st
            assert rel(x, xo) <= 1e-8
        else:
            assert st["iterations"] == 0 and rel(x, xo) <= 1e-10
        h.free()


@pytest.mark.parametrize("kind", ["fp16", "tf32"])
def test_two_block_passes_match_one_block_passes(gpu, monkeypatch, kind):
    """The outer update in two-block passes (the first block over the next block's columns,
    the second over the rest with both blocks' pivots, K up to 512) against one pass per
    block: the pivots agree to FP32 accumulation order (the pair sums both blocks in the
    accumulator before adding to the front), both refine to 1e-12, and the two-block
    factor matches the oracle."""
    model = W.hex8_cube(20).full()
    if kind == "tf32":
        monkeypatch.setenv("RFG_TC_KIND", "tf32")
    out = {}
    for pair in ("0", "1"):
        monkeypatch.setenv("RFG_TC_PAIR", pair)
        h, err, d = ffi.factor(model, precision=ffi.MIXED, want_d=True)
        assert h is not None, ffi.last_error()
        st0 = h.stats()
        x, st = h.solve(model.rhs, stats=True)
        assert st["backward_error"] <= 1e-12, (pair, st)
        out[pair] = (d, x, st0)
        h.free()
    d0, d1 = out["0"][0], out["1"][0]
    assert float(np.max(np.abs(d0 - d1) / np.abs(d0))) <= 1e-4
    # the pair passes update fewer entries with a longer K: the same flops, less traffic
    assert out["1"][2]["schur_entries"] < out["0"][2]["schur_entries"]
    ho, _, _ = refcpu.factor(model)
    assert rel(out["1"][1], ho.solve(model.rhs)) <= 1e-8
