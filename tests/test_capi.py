"""The C-ABI library loads and exports every function include/rustyfem_gpu.h
declares; host-side behaviour that needs no GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

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


def test_unsymmetric_invalid_input_is_refused_on_the_host():
    """rustyfem_factor_unsym validates like the other modes (ffi/src/lib.rs:101-104): -1."""
    m = W.chain(10, lambda c: 2.0, lambda r, c: -1.3 if r > c else -0.7)
    bad = W.Model(m.name, m.n, m.nn, m.loc.copy(), m.coords, m.indptr, m.indices, m.data, m.rhs, None, "full")
    bad.loc[3] = m.nn + 1
    h, err, _ = ffi.factor_unsym(bad)
    assert h is None and err == -1


def test_unsymmetric_without_a_device_fails_loudly():
    if ffi.device_count() > 0:
        pytest.skip("a CUDA device is present")
    m = W.chain(10, lambda c: 2.0, lambda r, c: -1.3 if r > c else -0.7)
    h, err, _ = ffi.factor_unsym(m)
    assert h is None and err == -1
    assert "no CUDA device" in ffi.last_error()


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


def test_timing_printout_format():
    """RUSTYFEM_TIMING: the engine-level prepare prints the reference's analysis line
    (src/solver/direct.rs:27-35) before it needs a device."""
    import subprocess
    import sys

    code = (
        "import numpy as np, ctypes\n"
        "from rustyfem_b200 import ffi, workloads as W\n"
        "g = W.hex8_cube(6).graph\n"
        "F, I = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)\n"
        "c = np.ascontiguousarray(g.coords, np.float64)\n"
        "m = ffi.lib().rfg_matrix_prepare(len(g.ndof), c.ctypes.data_as(F), g.adj_ptr.ctypes.data_as(I),\n"
        "    g.adj_idx.ctypes.data_as(I), g.ndof.ctypes.data_as(I), 0, 0)\n"
        "if m: ffi.lib().rfg_matrix_free(m)\n"
    )
    env = dict(os.environ, RUSTYFEM_TIMING="1")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    line = [ln for ln in out.stderr.splitlines() if ln.startswith("analysis:")][0]
    mt = re.fullmatch(r"analysis: \d+\.\d{3} s  flops: (\d\.\d\de-?\d+)  factor: (\d+) MB  largest front: "
                      r"\((\d+), (\d+)\)", line)
    assert mt, line
    sym = ffi.Symbolic(W.hex8_cube(6).graph, 48)
    assert mt.group(1) == ("%.2e" % sym.work()).replace("e+0", "e").replace("e+", "e")
    assert int(mt.group(2)) == (sym.factor_size() * 8) >> 20
    big = max(((int(k), int(u)) for _, k, u, _ in sym.fronts()), key=lambda t: t[0] + t[1])
    assert (int(mt.group(3)) + int(mt.group(4))) == sum(big)
