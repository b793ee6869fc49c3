"""rfg_solve_device_noalloc against rfg_solve_device.

The no-allocation entry point runs the same sweep kernels on a fixed device scratch
array instead of the handle's own buffers. With refinement off (refine_max_iter = 0,
no statistics) rfg_solve_device applies the factor once, so both must give the same
values bit for bit, on every call (the backward sweep's ticket counters live in the
shared scratch and must be back at zero for the next call). The call must take no
device memory, and a handle whose scratch need is above the fixed size is refused
before anything runs. This file is named to be collected last, so that it also runs
after every other GPU test has loaded and used the library.
"""
import ctypes

import numpy as np
import pytest

from rustyfem_b200 import ffi, workloads as W

pytestmark = pytest.mark.gpu


def _solve_device_plain(h, b, nrhs):
    """rfg_solve_device with stats = NULL: no refinement when refine_max_iter = 0."""
    rc = ffi.lib().rfg_solve_device(h.ptr, nrhs, ctypes.c_void_p(b.data_ptr()), None)
    assert rc == 0, ffi.last_error()


def _with_uncoupled(base, extra=4):
    """base plus `extra` diagonal-only DOFs (solved by division, not by the sweep)."""
    n0 = base.n
    n = n0 + extra
    indptr = np.concatenate([base.indptr, base.indptr[-1] + np.arange(1, extra + 1)])
    indices = np.concatenate([base.indices, np.arange(n0, n)])
    data = np.concatenate([base.data, np.linspace(2.0, 5.0, extra)])
    loc = np.concatenate([base.loc, np.zeros(extra, np.int64)])
    return W.Model(base.name + "+iso", n, base.nn, loc, base.coords, indptr, indices, data, np.ones(n), None, "full")


@pytest.mark.parametrize("precision", [ffi.FP64, ffi.MIXED])
@pytest.mark.parametrize("case,nrhs", [("plate", 3), ("cube_iso", 1), ("plate", 40)])
def test_same_values_as_solve_device_two_calls(gpu, precision, case, nrhs):
    import torch

    m = W.plate(60, 6).full() if case == "plate" else _with_uncoupled(W.hex8_cube(6).full())
    h, err, _ = ffi.factor(m, precision=precision, refine_max_iter=0)
    assert h is not None, ffi.last_error()
    rng = np.random.default_rng(7)
    try:
        for call in range(2):
            b = torch.from_numpy(rng.standard_normal((nrhs, m.n)) * 1e3).cuda()
            # the copies are queued on torch's current stream, the legacy default stream
            # here: both entry points make the handle's stream wait for it on entry
            assert torch.cuda.current_stream().cuda_stream == 0
            ref = b.clone()
            got = b.clone()
            _solve_device_plain(h, ref, nrhs)
            h.solve_device_noalloc(got.data_ptr(), nrhs)
            torch.cuda.synchronize()
            assert torch.equal(ref, got), f"call {call}: max diff {(ref - got).abs().max().item()}"
            if precision == ffi.FP64:
                x = got.cpu().numpy()
                r = np.array([m.matvec(x[j]) for j in range(nrhs)]) - b.cpu().numpy()
                assert np.linalg.norm(r) / np.linalg.norm(b.cpu().numpy()) < 1e-9
    finally:
        h.free()


def test_takes_no_device_memory(gpu):
    import torch

    m = W.plate(80, 8).full()
    h, _, _ = ffi.factor(m, refine_max_iter=0)
    assert h is not None, ffi.last_error()
    b = torch.from_numpy(np.random.default_rng(3).standard_normal((4, m.n))).cuda()
    try:
        h.solve_device_noalloc(b.data_ptr(), 4)  # set-up: scratch address, kernel attributes
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(3):
            h.solve_device_noalloc(b.data_ptr(), 4)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
    finally:
        h.free()


def test_refuses_beyond_the_fixed_scratch(gpu):
    import torch

    # 30³ C3D8 cube: 89 373 DOF; 32 right-hand sides need > 2 × 22 MB for X and Y alone
    m = W.hex8_cube(30).full()
    h, _, _ = ffi.factor(m, refine_max_iter=0)
    assert h is not None, ffi.last_error()
    b = torch.ones((32, m.n), dtype=torch.float64, device="cuda")
    try:
        with pytest.raises(RuntimeError, match="16777216 bytes"):
            h.solve_device_noalloc(b.data_ptr(), 32)
        torch.cuda.synchronize()
        assert bool((b == 1.0).all())  # nothing ran
        st = h.solve_device(b.data_ptr(), 32)  # the regular entry point solves it
        assert st["backward_error"] < 1e-12
    finally:
        h.free()
