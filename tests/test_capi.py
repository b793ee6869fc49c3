"""The C-ABI library loads and exports every function include/rustyfem_gpu.h
declares; host-side behaviour that needs no GPU."""
import ctypes
import os
import re

import numpy as np

from rustyfem_b200 import _build, ffi, workloads as W

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "rustyfem_gpu.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b((?:rustyfem|rfg)_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(_build.gpu_library())
    names = declared()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(ffi.EXPORTS) == names


def test_reference_symbols_present():
    """The eight functions of ffi/src/lib.rs keep their names."""
    names = declared()
    for n in ["rustyfem_factor", "rustyfem_factor_indef", "rustyfem_factor_unsym", "rustyfem_inertia",
              "rustyfem_solve", "rustyfem_info", "rustyfem_order", "rustyfem_free"]:
        assert n in names


def test_unsymmetric_is_refused_with_minus_one():
    m = W.chain(10, lambda c: 2.0, lambda r, c: -1.0)
    h, err = ffi.factor_unsym(m)
    assert h is None and err == -1
    assert "unsymmetric" in ffi.last_error()


def test_invalid_input_is_refused_on_the_host():
    m = W.hex8_cube(2).full()
    bad = W.Model(m.name, m.n, m.nn, m.loc.copy(), m.coords, m.indptr, m.indices, m.data, m.rhs, None, "full")
    bad.loc[0] = m.nn + 3
    h, err, _ = ffi.factor(bad)
    assert h is None and err == -1
    assert "loc" in ffi.last_error()


def test_uncoupled_nonpositive_dof_is_refused_on_the_host():
    n = 6
    m = W.Model("diag", n, n, np.arange(n), np.zeros(3 * n), np.arange(n + 1), np.arange(n),
                np.array([1.0, 2.0, 0.0, 4.0, 5.0, 6.0]), np.ones(n), None, "full")
    h, err, _ = ffi.factor(m)
    assert h is None and err == 2


def test_no_gpu_fails_loudly():
    """Without a CUDA device the factorization refuses (there is no CPU path)."""
    if ffi.device_count() > 0:
        return
    m = W.hex8_cube(2).full()
    h, err, _ = ffi.factor(m)
    assert h is None and err == -1
    assert "no CUDA device" in ffi.last_error()


def _fronts_dumped_by_prepare(model):
    """The front list rustyfem_factor prints under RUSTYFEM_FRONTS (ffi/src/lib.rs:163-167),
    read from the host stage alone: without a GPU the call then stops with an error."""
    import tempfile

    os.environ["RUSTYFEM_FRONTS"] = "1"
    fd = os.dup(2)
    try:
        with tempfile.TemporaryFile(mode="w+") as tmp:
            os.dup2(tmp.fileno(), 2)
            try:
                ffi.factor(model)
            finally:
                os.dup2(fd, 2)
            tmp.seek(0)
            lines = [ln.split()[1:] for ln in tmp.read().splitlines() if ln.startswith("front ")]
    finally:
        os.close(fd)
        del os.environ["RUSTYFEM_FRONTS"]
    return np.array(lines, np.int64).reshape(-1, 4)


def test_host_graph_from_the_pattern_matches_the_oracle():
    """The node graph prepare_model builds from the CSC pattern (both triangles or the
    lower one only) gives the oracle's front list (start, k, u, children)."""
    import pytest

    from oracle import refcpu

    if ffi.lib().rfg_device_count() > 0:
        pytest.skip("with a GPU the call factors the model instead of stopping after the host stage")
    for model in (W.hex8_cube(5), W.plate(30, 3), W.hex20_cube(3)):
        want = refcpu.Symbolic(model.graph, 16).fronts()
        for m in (model.full(), model):
            got = _fronts_dumped_by_prepare(m)
            assert np.array_equal(got, want), (m.name, m.symmetric_storage)
