"""The sweep workspace of a handle grows from four right-hand sides to 32 when a wider solve
comes; the sweeps captured for the narrower buffers are dropped and captured again. Solves
with one right-hand side before and after the growth give the same bits, and the wide solve
matches the narrow ones column by column (both refined to a backward error of 1e-12)."""
import numpy as np
import pytest

from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu


def test_workspace_grows_for_wider_solves(gpu):
    model = W.hex8_cube(12).full()
    h, err, _ = ffi.factor(model, precision=ffi.MIXED)
    assert h is not None, ffi.last_error()
    try:
        rng = np.random.default_rng(5)
        B = rng.standard_normal((8, model.n))
        x1 = [h.solve(B[0]) for _ in range(3)]  # direct, then captured, then replayed
        assert all(np.array_equal(x1[0], x) for x in x1[1:])
        X8 = h.solve(B)  # wider: the workspace grows
        x1b = [h.solve(B[0]) for _ in range(3)]
        assert all(np.array_equal(x1[0], x) for x in x1b)
        for j in range(8):
            xj = h.solve(B[j])
            assert float(np.linalg.norm(X8[j] - xj) / np.linalg.norm(xj)) <= 1e-8, j
    finally:
        h.free()
