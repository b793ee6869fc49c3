#!/usr/bin/env python
"""Benchmark: factor + solve of the 60³ C3D8 elasticity cube (n = 669,780 free DOFs)
on one B200, mixed precision + FP64 refinement to a normwise backward error of
1e-12, next to the plain FP64 GPU path.

One step = the numeric factorization of the cube's stiffness matrix (values
resident in HBM) followed by the solve of its load case with FP64 iterative
refinement until the backward error is at most 1e-12 (mixed) / a plain solve
(FP64). The symbolic stage is done once outside the timed region, as for a
Newton loop that refactors the same pattern.

  value    seconds per mixed-precision step, device-timed with CUDA events on
           the library's stream (max over ranks)
  e2e      the same step through the C interface with host buffers: rfg_factor_ex
           (analysis, plan, upload, factor) + rfg_solve_ex + rustyfem_free
  roofline the outer Schur-update kernel, device time of its launches (CUDA events
           around each launch) against the larger of two step bounds: its least HBM
           traffic (updated entries read and written once, operands read once) at
           the measured copy peak, and its executed MMA flops at the measured dense
           FP16 rate; both reported
  cpu_baseline  the oracle (CPU restatement of the reference's multithreaded
           multifrontal solver) factoring and solving the same 60³ cube once with
           all host threads; its solution is the reference for rel_err_vs_oracle
  c3b      the same cube with per-element E log-uniform in [1e3, 1e9] Pa (seed 0):
           both GPU paths, refinement iterations, backward error and the relative
           error against the oracle's solution
  plates, hex20, indefinite, assembly, unsymmetric  the batched 512-plate case, the
           40³ C3D20 cube with 32 right-hand sides, the shifted (indefinite) 30³ cube through
           rustyfem_factor_indef, the assembly of the 60³ cube's K on the GPU against the
           oracle's element loop, and the skewed 24³ cube through rustyfem_factor_unsym
           (skipped with --no-extras)

``--impl reference`` times the reference's CPU algorithm (the oracle port: the
reference is Rust and cannot be built here) on the same workload: its K timed
steps together run one whole factor + solve of the cube (analysis, the
elimination tree bottom-up by depth, the solve), so that every step is a bounded
slice and the sum is a measured time of the full workload.
Multi-GPU: the single model does not shard; --gpus N runs N replicas (one per
rank), and value is the slowest rank's step time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Factor+solve s, mixed-prec vs FP64 LDLᵀ on B200 at backward err ≤1e-12"
WORKLOAD_N = 60
REF_FACTOR_PARTS = 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--n", type=int, default=WORKLOAD_N, help="cube size (elements per edge)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in small/large-front cutover instead of tuning it on the workload")
    ap.add_argument("--no-oracle", action="store_true",
                    help="skip the oracle (CPU) factor + solve of the workload: no cpu_baseline, no rel_err_vs_oracle")
    ap.add_argument("--no-c3b", action="store_true", help="skip the log-uniform-E variant of the cube")
    ap.add_argument("--no-extras", action="store_true", help="skip the plates and hex20 sub-records")
    ap.add_argument("--workload", choices=["hex8", "hex20", "plates", "indef", "assembly", "unsym"], default="hex8",
                    help="hex8: the 60³ C3D8 cube (default, the headline); hex20: the 40³ C3D20 cube with 32 "
                         "right-hand sides; plates: 512 CPS4 plates with 8 right-hand sides each, batched; "
                         "indef: the shifted cube through the indefinite path; assembly: K of the n³ cube "
                         "assembled on the GPU; unsym: the skewed n³ cube through the unsymmetric LU")
    ap.add_argument("--profile-precision", choices=["mixed", "fp64", "both"], default="both",
                    help="--profile-only: which factorizations to run")
    ap.add_argument("--profile-only", action="store_true",
                    help="only factor (twice more) and solve the n³ cube in both precisions: the target of ncu captures")
    return ap.parse_args()


def workload_config(n: int, model, flops: float, nfronts: int) -> dict:
    """The workload description both arms print (the driver compares the two)."""
    return {"workload": f"hex8 {n}^3 C3D8 elasticity (n={model.n} free DOFs, nnz(A, both triangles)={model.nnz}): "
                        "numeric factorization + solve of the load case",
            "leaf": 16, "nrhs": 1, "flops": int(round(flops)), "nfronts": int(nfronts),
            "l2": "inputs larger than L2 (the factor and the fronts take GBs)"}


def _device_step_seconds(torch, h, data_d, b_d, rhs_d, nrhs, steps, warmup):
    """Device time (CUDA events on the library's stream) of refactor + refined solve."""
    from rustyfem_b200 import ffi

    stream = torch.cuda.ExternalStream(h.stream())
    last = None
    tot = 0.0
    for it in range(warmup + steps):
        b_d.copy_(rhs_d)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if h.refactor_device(data_d.data_ptr()) != -1:
            raise RuntimeError("refactor failed: " + ffi.last_error())
        last = h.solve_device(b_d.data_ptr(), nrhs)
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= warmup:
            tot += e0.elapsed_time(e1) / 1e3
    return tot / steps, last


def measure_hex20(n: int, steps: int, warmup: int) -> dict:
    """The n³ C3D20 cube with 32 seeded normal right-hand sides, mixed precision with
    FP64 refinement, and the FP64 path beside it (device time per step)."""
    import numpy as np
    import torch

    from rustyfem_b200 import ffi, workloads as W

    m = W.hex20_cube(n).full().with_rhs(32, seed=0)
    data_d = torch.from_numpy(m.data).cuda()
    rhs_d = torch.from_numpy(np.ascontiguousarray(m.rhs)).cuda()
    b_d = torch.empty_like(rhs_d)
    out = {}
    for name, prec in (("mixed", ffi.MIXED), ("fp64", ffi.FP64)):
        h, err, _ = ffi.factor(m, precision=prec, refine_tol=1e-12)
        if h is None:
            raise RuntimeError(ffi.last_error())
        sec, st = _device_step_seconds(torch, h, data_d, b_d, rhs_d, 32, steps, warmup)
        fst = h.stats()
        out[name] = {"s": sec, "flops": fst["work"], "tflops": fst["work"] / sec / 1e12,
                     "iterations": st["iterations"], "backward_error": st["backward_error"],
                     "rel_residual": st["rel_residual"]}
        h.free()
    del data_d, rhs_d, b_d
    torch.cuda.empty_cache()
    return {"workload": f"hex20 {n}^3 C3D20 (n={m.n}), 32 seeded normal right-hand sides", "unit": "s",
            "steps": steps, "warmup": warmup, "mixed": out["mixed"], "fp64": out["fp64"],
            "speedup_mixed_vs_fp64": out["fp64"]["s"] / out["mixed"]["s"]}


def measure_plates(steps: int, warmup: int) -> dict:
    """512 CPS4 cantilever plates (nx ~ U{20..200}, ny = max(2, nx/10)), 8 right-hand
    sides each: the batched factorization (one CUDA graph) + solve against the same
    plates factored and solved one by one through the same library. Both sides are
    given as device time (CUDA events on the handles' streams) and as host wall time
    (each from its first launch to the synchronize after its last)."""
    import numpy as np
    import torch

    from rustyfem_b200 import ffi, workloads as W

    models = [mm.full() for mm in W.plate_batch(512, seed=0, nrhs=8)]
    out = {}
    for name, prec in (("fp64", ffi.FP64), ("mixed", ffi.MIXED)):
        bh, em, ed = ffi.factor_batch(models, precision=prec, refine_tol=1e-12)
        if bh is None:
            raise RuntimeError(ffi.last_error())
        data = np.concatenate([mm.data for mm in models])
        rhs = bh.stack([mm.rhs for mm in models])
        data_d = torch.from_numpy(data).cuda()
        rhs_d = torch.from_numpy(np.ascontiguousarray(rhs)).cuda()
        b_d = torch.empty_like(rhs_d)
        sec, st = _device_step_seconds(torch, bh, data_d, b_d, rhs_d, 8, steps, warmup)
        walls = []
        for _ in range(steps):
            b_d.copy_(rhs_d)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            bh.refactor_device(data_d.data_ptr())
            bh.solve_device(b_d.data_ptr(), 8)
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
        fst = bh.stats()
        # the same plates one by one: per plate the numeric phase and the 8-RHS solve on
        # device-resident data, device time from events on the plate handle's stream
        per = []
        for mm in models:
            h = ffi.factor(mm, precision=prec, refine_tol=1e-12)[0]
            dd = torch.from_numpy(mm.data).cuda()
            rr = torch.from_numpy(np.ascontiguousarray(mm.rhs)).cuda()
            per.append((h, dd, rr, torch.empty_like(rr)))
        for h, dd, rr, bb in per:  # warm-up (graph capture on the second numeric phase)
            for _ in range(2):
                h.refactor_device(dd.data_ptr())
                bb.copy_(rr)
                h.solve_device(bb.data_ptr(), 8)
        torch.cuda.synchronize()
        dev = 0.0
        t0 = time.perf_counter()
        for h, dd, rr, bb in per:
            bb.copy_(rr)
            stream = torch.cuda.ExternalStream(h.stream())
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h.refactor_device(dd.data_ptr())
            h.solve_device(bb.data_ptr(), 8)
            e1.record(stream)
            e1.synchronize()
            dev += e0.elapsed_time(e1) / 1e3
        wall_one = time.perf_counter() - t0
        for h, *_ in per:
            h.free()
        del per
        out[name] = {"batched_s": sec, "batched_wall_s": statistics.median(walls),
                     "batched_factor_ms": fst["t_factor_ms"], "launches_in_graph": fst["launches"],
                     "nfronts": fst["nfronts"], "levels": fst["nlevels"],
                     "one_by_one_device_s": dev, "one_by_one_wall_s": wall_one,
                     "speedup_device": dev / sec, "speedup_wall": wall_one / statistics.median(walls),
                     "iterations": st["iterations"], "backward_error": st["backward_error"],
                     "rel_residual": st["rel_residual"]}
        bh.free()
        del data_d, rhs_d, b_d
        torch.cuda.empty_cache()
    # the per-model precision choice (RFG_AUTO) on this batch
    ba, _, _ = ffi.factor_batch(models, precision=ffi.AUTO, refine_tol=1e-12)
    auto = {0: "fp64", 1: "mixed"}.get(int(ba.stats()["precision"]))
    ba.free()
    return {"workload": "512 CPS4 plates (nx ~ U{20..200}, ny = max(2, nx/10), seed 0), 8 right-hand sides each",
            "unit": "s", "steps": steps, "warmup": warmup, **out, "auto_precision_choice": auto,
            "basis": "speedup_device: sum over plates of the device time of refactor + solve (CUDA events per plate) "
                     "over the batched device time; speedup_wall: host wall time of the one-by-one loop over the "
                     "batched call's"}


def shifted_cube(n: int, frac: float = 0.2):
    """The n³ C3D8 cube with frac × the median diagonal subtracted from the diagonal: an
    indefinite system with 1×1 and 2×2 pivots and delayed pivots."""
    import numpy as np

    from rustyfem_b200 import workloads as W

    m = W.hex8_cube(n).full()
    d = m.data.copy()
    pos = np.array([m.indptr[c] + int(np.where(m.indices[m.indptr[c]:m.indptr[c + 1]] == c)[0][0])
                    for c in range(m.n)])
    d[pos] -= frac * float(np.median(d[pos]))
    return W.Model(m.name + " shifted", m.n, m.nn, m.loc, m.coords, m.indptr, m.indices, d, m.rhs, None, "full")


def measure_indef(n: int, oracle: bool) -> dict:
    """The symmetric indefinite path (rustyfem_factor_indef + rustyfem_solve) on the n³ cube
    shifted into the indefinite range: wall time of the C-interface calls, inertia, and the
    comparison with the oracle."""
    import numpy as np

    from rustyfem_b200 import ffi

    ms = shifted_cube(n)
    h, err, ine = ffi.factor_indef(ms)  # first call: loads kernels, fills the memory pools
    if h is None:
        raise RuntimeError(f"indefinite factorization failed at {err}: {ffi.last_error()}")
    h.free()
    t0 = time.perf_counter()
    h, err, ine = ffi.factor_indef(ms)
    t1 = time.perf_counter()
    x = h.solve(ms.rhs)
    t2 = time.perf_counter()
    h.free()
    rec = {"workload": f"hex8 {n}^3 C3D8 with 0.2 x the median diagonal subtracted (n={ms.n}), indefinite",
           "factor_call_s": t1 - t0, "solve_call_s": t2 - t1, "inertia": list(ine)}
    if oracle:
        from oracle import refcpu

        t0 = time.perf_counter()
        ho, erro, ineo = refcpu.factor_indef(ms)
        xo = ho.solve(ms.rhs)
        rec["oracle_s"] = time.perf_counter() - t0
        rec["oracle_inertia"] = list(ineo)
        rec["inertia_equal"] = tuple(ine) == tuple(ineo)
        rec["rel_err_vs_oracle"] = float(np.linalg.norm(x - xo) / np.linalg.norm(xo))
        ho.free()
    return rec


def measure_assembly(n: int, oracle: bool) -> dict:
    """Assembly of K on the GPU (rfg_assembly_hex8: the C3D8 element matrices on the device, then
    each lower entry summed from its element contributions in the reference's order) for the
    n³ cube, against the oracle's restatement of the reference's element loop (element matrices
    in parallel blocks, then added one element after another) on the host threads."""
    import numpy as np

    from rustyfem_b200 import solver, workloads as W

    m = W.hex8_cube(n)
    me = W.hex8_mesh(n)
    sm = solver.select("direct-gpu-mixed").prepare(m.graph)
    edof = me.edof(sm.first_dof())
    t0 = time.perf_counter()
    asm = sm.assembly(edof)
    t_prep = time.perf_counter() - t0
    asm.hex8(me.xyz, me.conn, me.emod, me.nu)  # first call: allocations
    el, ga, wall = [], [], []
    for _ in range(5):
        t0 = time.perf_counter()
        asm.hex8(me.xyz, me.conn, me.emod, me.nu)
        wall.append(time.perf_counter() - t0)
        a, b = asm.times()
        el.append(a)
        ga.append(b)
    nc = asm.contributions()
    nnz = sm.nnz()
    g_ms = statistics.median(ga)
    # the gather's least traffic: each key read (8 B), both element-matrix values of a
    # contribution (2 × 8 B), the entry's start (8 B) and its value written (8 B)
    g_bytes = 24.0 * nc + 16.0 * nnz
    rec = {"workload": f"hex8 {n}^3 C3D8 stiffness (n={sm.n()}, {len(me.conn)} elements, {nnz} lower entries, "
                       f"{nc} element contributions)",
           "prepare_s": t_prep, "element_kernel_ms": statistics.median(el), "gather_ms": g_ms,
           "call_s": statistics.median(wall),
           "gather_gbs": g_bytes / (g_ms / 1e3) / 1e9 if g_ms > 0 else None,
           "note": "prepare maps the element pairs onto the pattern once per mesh; call = rfg_assembly_hex8 "
                   "(coordinates, connectivity and E uploaded, element kernel, gather), wall time"}
    if oracle:
        from oracle import refcpu

        sym = refcpu.Symbolic(m.graph, 48)
        colptr, rowidx = sym.pattern()
        t0 = time.perf_counter()
        vo = refcpu.assemble_hex8(colptr, rowidx, me.conn, me.xyz, me.emod, me.nu, edof)
        rec["oracle_s"] = time.perf_counter() - t0
        rec["oracle_threads"] = refcpu.threads()
        rec["bit_identical_to_oracle"] = bool(np.array_equal(sm.values(), vo))
        rec["speedup_call_vs_oracle"] = rec["oracle_s"] / rec["call_s"]
    del asm
    return rec


def measure_unsym(n: int, oracle: bool) -> dict:
    """The unsymmetric LU path (rustyfem_factor_unsym + rustyfem_solve) on the n³ cube with a
    strong skew-symmetric part (diagonals fail the threshold test, pivots are delayed): wall time
    of the C-interface calls, delayed pivots, and the comparison with the oracle."""
    import numpy as np

    from rustyfem_b200 import ffi, workloads as W

    m = W.skew_perturbed(W.hex8_cube(n), 30.0, seed=0)
    h, err, st = ffi.factor_unsym(m)  # first call: loads kernels, fills the memory pools
    if h is None:
        raise RuntimeError(f"LU factorization failed at {err}: {ffi.last_error()}")
    h.free()
    t0 = time.perf_counter()
    h, err, st = ffi.factor_unsym(m)
    t1 = time.perf_counter()
    x = h.solve(m.rhs)
    t2 = time.perf_counter()
    rec = {"workload": f"hex8 {n}^3 C3D8 plus a skew-symmetric part of 30 x the largest diagonal (n={m.n}), "
                       "unsymmetric LU", "factor_call_s": t1 - t0, "solve_call_s": t2 - t1,
           "delayed": int(st["delayed"]), "factor_size": int(h.info()[1])}
    h.free()
    if oracle:
        from oracle import refcpu

        t0 = time.perf_counter()
        ho, erro, dlo = refcpu.factor_unsym(m)
        xo = ho.solve(m.rhs)
        rec["oracle_s"] = time.perf_counter() - t0
        rec["oracle_delayed"] = dlo
        rec["delayed_equal"] = dlo == rec["delayed"]
        rec["rel_err_vs_oracle"] = float(np.linalg.norm(x - xo) / np.linalg.norm(xo))
        ho.free()
    return rec


def run_hex20(args):
    n = 40 if args.n == WORKLOAD_N else args.n
    print(json.dumps(measure_hex20(n, args.steps, args.warmup)), flush=True)


def run_plates(args):
    print(json.dumps(measure_plates(args.steps, args.warmup)), flush=True)


def run_profile_case(args):
    """A short, fixed sequence of the library's kernels for profiler captures."""
    from rustyfem_b200 import ffi, workloads as W

    m = W.hex8_cube(args.n).full()
    cases = {"mixed": [(ffi.MIXED, True)], "fp64": [(ffi.FP64, False)], "both": [(ffi.MIXED, True), (ffi.FP64, False)]}
    for prec, tc in cases[args.profile_precision]:
        h, err, _ = ffi.factor(m, precision=prec, tensor_cores=tc, refine_tol=1e-12)
        if h is None:
            raise RuntimeError(ffi.last_error())
        for _ in range(2):
            if h.refactor(m.data) != -1:
                raise RuntimeError(ffi.last_error())
        x, st = h.solve(m.rhs, stats=True)
        print(json.dumps({"precision": prec, "t_factor_ms": h.stats()["t_factor_ms"], **st}), flush=True)
        h.free()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.path or not os.path.exists(self.path):
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


# ---------------------------------------------------------------------------
# measured peaks for the roofline denominators
# ---------------------------------------------------------------------------
def measure_peaks(torch):
    """cuBLAS FP64 and FP32 (no TF32) GEMM throughput on this GPU, best of 5."""
    out = {}
    n = 8192
    for name, dt, tf32 in [("fp64_tflops", torch.float64, False), ("fp32_tflops", torch.float32, False),
                           ("tf32_tflops", torch.float32, True)]:
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, device="cuda", dtype=dt)
        b = torch.randn(n, n, device="cuda", dtype=dt)
        for _ in range(2):
            a @ b
        best = 1e9
        for _ in range(5):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            a @ b
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        out[name] = 2 * n ** 3 / best / 1e12
        del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.cuda.empty_cache()
    return out


def read_peaks_file():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def read_traffic(kernel: str):
    """Measured DRAM bytes per byte of least traffic of a kernel, from its committed ncu
    summary (the capture's dram__bytes_read.sum + dram__bytes_write.sum over the least
    traffic of the captured launches), or None. The bench scales it by the least traffic of
    one launch."""
    path = os.path.join(HERE, "profiles", f"{kernel}_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_least_byte:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------
# CPU baseline: the oracle
# ---------------------------------------------------------------------------
def oracle_solve(model) -> dict:
    """Factor + solve of ``model`` by the oracle (the CPU restatement of the reference's
    multithreaded multifrontal solver) with all host threads, timed in its three parts:
    the analysis of rustyfem_factor, the numeric factorization, the solve."""
    from oracle import refcpu

    refcpu.set_threads(0)
    t0 = time.perf_counter()
    S = refcpu.StagedFactor(model, 1)
    t1 = time.perf_counter()
    ok = S.part(0)
    t2 = time.perf_counter()
    h, err = S.finish()
    if not ok or h is None:
        raise RuntimeError(f"oracle factorization failed at DOF {err}")
    x = h.solve(model.rhs)
    t3 = time.perf_counter()
    work, _ = h.info()
    nfronts = len(h.fronts())
    h.free()
    return {"x": x, "analysis_s": t1 - t0, "factor_s": t2 - t1, "solve_s": t3 - t2, "cores": refcpu.threads(),
            "flops": work, "nfronts": nfronts}


def rel_err(x, xo) -> float:
    import numpy as np

    return float(np.linalg.norm(x - xo) / np.linalg.norm(xo))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def c3b_record(n: int, steps: int, warmup: int, autotune: bool) -> tuple[dict, "object", dict]:
    """The cube with per-element E = 10^U(3, 9) Pa (numpy PCG64 seed 0): device step
    time of both GPU paths, refinement iterations, backward errors and the solutions
    (for the comparison with the oracle)."""
    import numpy as np
    import torch

    from rustyfem_b200 import ffi, workloads as W

    mb = W.hex8_cube(n, emod=W.log_uniform_moduli(n, seed=0)).full()
    data_d = torch.from_numpy(mb.data).cuda()
    rhs_d = torch.from_numpy(mb.rhs).cuda()
    b_d = torch.empty_like(rhs_d)
    rec, xs = {}, {}
    for name, prec in (("mixed", ffi.MIXED), ("fp64", ffi.FP64)):
        h, err, _ = ffi.factor(mb, precision=prec, refine_tol=1e-12, autotune=autotune)
        if h is None:
            raise RuntimeError(f"c3b factorization failed ({name}) at {err}: {ffi.last_error()}")
        sec, st = _device_step_seconds(torch, h, data_d, b_d, rhs_d, 1, steps, warmup)
        x, st2 = h.solve(mb.rhs, stats=True)
        xs[name] = x
        rec[name] = {"s": sec, "iterations": st2["iterations"], "backward_error": st2["backward_error"],
                     "rel_residual": st2["rel_residual"]}
        h.free()
    del data_d, rhs_d, b_d
    torch.cuda.empty_cache()
    rec["speedup_mixed_vs_fp64"] = rec["fp64"]["s"] / rec["mixed"]["s"]
    rec["workload"] = (f"hex8 {n}^3 C3D8, per-element E log-uniform in [1e3, 1e9] Pa (numpy PCG64 seed 0), nu=0.3 "
                       f"(n={mb.n})")
    rec["steps"] = steps
    rec["warmup"] = warmup
    return rec, mb, xs


def run_b200(args, rank, world, local_rank):
    import numpy as np
    import torch

    torch.cuda.set_device(local_rank)
    from rustyfem_b200 import ffi, workloads as W

    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist = dist_mod
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(v):
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    model = W.hex8_cube(args.n).full()
    data_d = torch.from_numpy(model.data).cuda()
    rhs_d = torch.from_numpy(model.rhs).cuda()
    b_d = torch.empty_like(rhs_d)

    handles = {}
    tuning = {}
    for name, prec in [("mixed", ffi.MIXED), ("fp64", ffi.FP64)]:
        h, err, _ = ffi.factor(model, precision=prec, refine_tol=1e-12, autotune=not args.no_autotune)
        if h is None:
            raise RuntimeError(f"factorization failed ({name}) at {err}: {ffi.last_error()}")
        # inside the timed steps: CUDA events around the 128-tile outer updates only (the
        # roofline's kernel); an event after every launch would break the launches'
        # programmatic overlap and lengthen the step
        h.set_profiling(2)
        handles[name] = h
        tuning[name] = {"tile_cutover_rows": h.stats()["tile_cutover_rows"],
                        "measured_ms": {str(c): round(ms, 3) for c, ms in h.tune_report()}}

    def step(h):
        e = h.refactor_device(data_d.data_ptr())
        if e != -1:
            raise RuntimeError(f"refactor failed: {e} {ffi.last_error()}")
        b_d.copy_(rhs_d)
        torch.cuda.synchronize()
        return h.solve_device(b_d.data_ptr(), 1)

    results = {}
    for name in ("mixed", "fp64"):
        h = handles[name]
        for _ in range(args.warmup):
            step(h)
    barrier()
    clocks = ClockSampler(local_rank)
    with clocks:
        for name in ("mixed", "fp64"):
            h = handles[name]
            stream = torch.cuda.ExternalStream(h.stream())
            tot = 0.0
            schur_ms = 0.0
            schur_fl = 0.0
            schur_n = 0
            launches = 0
            slaunches = 0
            last = None
            barrier()
            for _ in range(args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                last = step(h)
                e1.record(stream)
                torch.cuda.synchronize()
                tot += e0.elapsed_time(e1) / 1e3
                st = h.stats()
                schur_ms += st["schur_ms"]
                schur_fl += st["schur_flops"]
                schur_n += st["schur_launches"]
                launches += st["launches"]
                slaunches += last["launches"]
            barrier()
            results[name] = dict(s=allmax(tot / args.steps), schur_ms=schur_ms / args.steps,
                                 schur_flops=schur_fl / args.steps, schur_launches=schur_n / args.steps,
                                 factor_launches=launches / args.steps, solve_launches=slaunches / args.steps,
                                 solve=last)
    clk = clocks.summary()
    # the phase breakdown from a profiling pass after the timed steps (an event after every
    # launch: phases a little longer than inside the timed steps)
    for name in ("mixed", "fp64"):
        h = handles[name]
        h.set_profiling(1)
        for _ in range(2):
            step(h)
        ph = h.stats()["phase_ms"]
        results[name]["phase_ms"] = dict(zip(["assembly", "extend_add", "pivot_blocks", "panels", "inner_updates",
                                              "outer_updates_64tiles", "outer_updates_128tiles"], ph))
        results[name]["phase_ms"]["note"] = "one factorization with an event after every launch, after the timed steps"
        h.set_profiling(0)
    stats_m = handles["mixed"].stats()
    for h in handles.values():
        h.free()
    del data_d, rhs_d, b_d
    torch.cuda.empty_cache()

    # e2e through the C interface with host buffers
    e2e = {}
    xs = {}
    for name, prec in [("mixed", ffi.MIXED), ("fp64", ffi.FP64)]:
        times = []
        parts = []
        h2d = d2h = 0
        # one untimed call first (as the timed steps have their warm-up): it fills the
        # library's device-memory pool that the following calls reuse
        hw, _, _ = ffi.factor(model, precision=prec, refine_tol=1e-12)
        hw.solve(model.rhs, stats=True)
        hw.free()
        for _ in range(args.e2e_steps):
            barrier()
            t0 = time.perf_counter()
            h, err, _ = ffi.factor(model, precision=prec, refine_tol=1e-12)
            t1 = time.perf_counter()
            x, st = h.solve(model.rhs, stats=True)
            t2 = time.perf_counter()
            fst = h.stats()
            h.free()
            t3 = time.perf_counter()
            times.append(t3 - t0)
            parts.append({"factor_call_s": t1 - t0, "host_analysis_plan_upload_s": fst["t_analyse_ms"] / 1e3,
                          "solve_call_s": t2 - t1, "free_s": t3 - t2, "iterations": st["iterations"],
                          "backward_error": st["backward_error"]})
            h2d = fst["h2d_bytes"] + model.n * 8
            d2h = model.n * 8 + fst["nfronts"] * 8
            xs[name] = x
        e2e[name] = dict(s=allmax(statistics.median(times)), h2d=h2d, d2h=d2h, parts=parts[-1])

    extras = {}
    c3b = None
    if rank == 0 and world == 1:
        if not args.no_c3b:
            c3b, model_b, xs_b = c3b_record(args.n, 3, 1, not args.no_autotune)
        if not args.no_extras:
            extras["plates"] = measure_plates(3, 1)
            extras["hex20"] = measure_hex20(40 if args.n == WORKLOAD_N else max(4, args.n * 2 // 3), 2, 1)
            extras["indefinite"] = measure_indef(30 if args.n == WORKLOAD_N else max(4, args.n // 2),
                                                 not args.no_oracle)
            extras["assembly"] = measure_assembly(args.n, not args.no_oracle)
            extras["unsymmetric"] = measure_unsym(24 if args.n == WORKLOAD_N else max(4, args.n // 3),
                                                  not args.no_oracle)

    out = None
    if rank == 0:
        peaks = measure_peaks(torch)
        filepk = read_peaks_file()
        mixed, fp64 = results["mixed"], results["fp64"]
        # The dominant kernel of the headline (mixed) path: the outer Schur update of the large
        # fronts on the tensor cores. Two bounds per step: its least HBM traffic (each updated
        # trailing entry read and written once, each operand value read once) at the measured
        # copy rate, and its executed MMA flops (three FP16 MMAs per multiply-add of the split)
        # at the measured dense FP16/BF16 rate. Passes of one outer block (K = 256: 64 flop/B,
        # 192 executed) sit below the machine balance of 251 flop/B and are HBM-bound; the
        # second pass of a two-block pair (K = 512: 128 flop/B, 384 executed) is above it. The
        # line's roofline is the larger of the two step bounds; both are reported.
        st_m = stats_m
        alg = mixed["schur_flops"] / (mixed["schur_ms"] / 1e3) / 1e12 if mixed["schur_ms"] > 0 else None
        hbm = filepk.get("hbm_gbs")
        bf16 = filepk.get("bf16_tflops")
        hbm_src = "MEASURED_PEAKS.json hbm_gbs (STREAM-style copy); of measured" if hbm else "fallback 6650 GB/s"
        if hbm is None:
            hbm = 6650.0
        if bf16 is None:
            bf16 = 1590.0
        alg_bytes = 8.0 * st_m["schur_entries"] + 4.0 * st_m["schur_opvals"]
        gbs = alg_bytes / (mixed["schur_ms"] / 1e3) / 1e9 if mixed["schur_ms"] > 0 else None
        # step bounds (ms) of the outer update: least traffic at the copy rate, executed MMA
        # flops at the dense rate
        t_hbm = alg_bytes / (hbm * 1e9) * 1e3
        t_tc = 3.0 * mixed["schur_flops"] / (bf16 * 1e12) * 1e3
        tc_bound = t_tc > t_hbm
        split_peak = bf16 / 3.0  # algorithmic rate of the split at the dense MMA rate
        ach64 = fp64["schur_flops"] / (fp64["schur_ms"] / 1e3) / 1e12 if fp64["schur_ms"] > 0 else None
        nl = max(mixed["schur_launches"], 1)
        ratio = read_traffic("schur_tc_persistent")
        traffic = ratio * alg_bytes / nl if ratio else None
        cpu = None
        orc = {}
        if not args.no_oracle and world == 1:
            o = oracle_solve(model)
            cpu = {"value": o["factor_s"] + o["solve_s"], "unit": "s", "cores": o["cores"], "kind": "port",
                   "sample": f"the whole workload: one factor + solve of the hex8 {args.n}^3 cube by the oracle "
                             f"(C++ restatement of the reference's threaded multifrontal LDLT) with {o['cores']} "
                             "host threads, measured once; value = numeric factorization + solve, as this line's "
                             "value",
                   "analysis_s": o["analysis_s"], "factor_s": o["factor_s"], "solve_s": o["solve_s"],
                   "with_analysis_s": o["analysis_s"] + o["factor_s"] + o["solve_s"]}
            orc["mixed"] = rel_err(xs["mixed"], o["x"])
            orc["fp64"] = rel_err(xs["fp64"], o["x"])
            del o
            if c3b is not None:
                ob = oracle_solve(model_b)
                c3b["mixed"]["rel_err_vs_oracle"] = rel_err(xs_b["mixed"], ob["x"])
                c3b["fp64"]["rel_err_vs_oracle"] = rel_err(xs_b["fp64"], ob["x"])
                c3b["oracle_factor_solve_s"] = ob["factor_s"] + ob["solve_s"]
                del ob
        if c3b is not None:
            c3b["mixed"]["rel_err_vs_fp64_gpu"] = rel_err(xs_b["mixed"], xs_b["fp64"])
        out = {
            "metric": METRIC,
            "value": mixed["s"],
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": mixed["s"] * 1e3,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 fronts, tensor-core Schur updates on the FP16 split of U = L D^(1/2) with power-of-two "
                     "row scales and f32 accumulation, f64 pivot blocks, D, residual and refinement",
            "data": "synthetic: 60^3 C3D8 unit cube, steel E=210e9 nu=0.3, x=0 clamped, fz=-1000 N on x=1",
            "config": workload_config(args.n, model, stats_m["work"], stats_m["nfronts"]),
            "parallelism": f"replicas x{world}",
            "autotune": tuning,
            "fp64": {"s": fp64["s"], "speedup_mixed_vs_fp64": fp64["s"] / mixed["s"],
                     "backward_error": fp64["solve"]["backward_error"],
                     "rel_err_vs_oracle": orc.get("fp64"),
                     "schur_tflops": ach64, "factor_tflops": stats_m["work"] / fp64["s"] / 1e12},
            "mixed": {"tc_kind": {0: "none", 1: "tf32 split", 2: "fp16 split of U = L D^(1/2), power-of-two row scales"}
                      .get(int(stats_m.get("tc_kind", 0))),
                      "iterations": mixed["solve"]["iterations"], "backward_error": mixed["solve"]["backward_error"],
                      "rel_residual": mixed["solve"]["rel_residual"], "rel_err_vs_oracle": orc.get("mixed"),
                      "rel_err_vs_fp64_gpu": rel_err(xs["mixed"], xs["fp64"]),
                      "factor_tflops": stats_m["work"] / mixed["s"] / 1e12},
            "c3b": c3b,
            "e2e": {"value": e2e["mixed"]["s"], "unit": "s", "h2d_bytes_per_step": e2e["mixed"]["h2d"],
                    "d2h_bytes_per_step": e2e["mixed"]["d2h"], "fp64_s": e2e["fp64"]["s"],
                    "speedup_mixed_vs_fp64": e2e["fp64"]["s"] / e2e["mixed"]["s"],
                    "last_step_parts": e2e["mixed"]["parts"], "fp64_last_step_parts": e2e["fp64"]["parts"],
                    "path": "rfg_factor_ex (host analysis + plan + upload + factor) + rfg_solve_ex + rustyfem_free, "
                            "after one untimed call of the same sequence"},
            "roofline": {"kernel": "k_schur_tc_persistent<256, FP16 split> (outer Schur update of the large fronts: "
                                   "tcgen05 kind::f16 on the FP16 head and tail of U = L D^(1/2) with power-of-two "
                                   "row scales, three MMAs per K step, two TMEM accumulators, TMA loads, TMA "
                                   "reduce-add into the front, warp-specialised)",
                         "bound": "tensor" if tc_bound else "hbm",
                         "achieved": alg if tc_bound else gbs,
                         "peak": split_peak if tc_bound else hbm,
                         "unit": "TFLOP/s" if tc_bound else "GB/s",
                         "frac": ((alg / split_peak) if tc_bound else (gbs / hbm)) if (alg and gbs) else None,
                         "achieved_basis": ("algorithmic flops of the outer-update launches per step (2K per "
                                            "updated trailing entry, from the plan) / their device time (CUDA events "
                                            "on the library stream, in the timed steps)") if tc_bound else
                                           ("least traffic of the outer-update launches per step (each updated "
                                            "trailing entry read and written once in FP32, 8 B; each operand value "
                                            "of the FP16 split read once, 4 B, from the plan) / their device time "
                                            "(CUDA events on the library stream, in the timed steps)"),
                         "peak_source": ("MEASURED_PEAKS.json bf16_tflops / 3: the split's three FP16 MMAs per "
                                         "multiply-add at the measured dense rate; of measured") if tc_bound
                                        else hbm_src,
                         "step_bounds_ms": {"hbm_least_traffic": t_hbm, "tensor_executed": t_tc,
                                            "measured": mixed["schur_ms"],
                                            "frac_of_larger": max(t_hbm, t_tc) / mixed["schur_ms"]
                                            if mixed["schur_ms"] > 0 else None},
                         "hbm": {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": (gbs / hbm) if gbs else None,
                                 "peak_source": hbm_src},
                         "traffic": traffic,
                         "traffic_basis": "dram__bytes_read.sum + dram__bytes_write.sum of three large launches of "
                                          "this kernel on the 40^3 cube (ncu) over their least traffic, times the "
                                          "least traffic of one launch here (profiles/schur_tc_persistent_traffic.txt)",
                         "alg_bytes_per_step": alg_bytes,
                         "why_bound": "arithmetic intensity 2K flops per 8-byte read-and-write of a trailing "
                                      "entry: 64 flop/B (192 executed) for a one-block pass (K = 256), 128 (384) for "
                                      "the second pass of a two-block pair (K = 512), against a machine balance of "
                                      "%.0f flop/B (FP16 dense %.1f TFLOP/s / HBM %.0f GB/s); the step's larger "
                                      "bound is the %s one" % (bf16 * 1e3 / hbm, bf16, hbm,
                                                                "tensor" if tc_bound else "HBM"),
                         "tensor": {"algorithmic_tflops": alg, "peak": bf16, "unit": "TFLOP/s",
                                    "frac": (alg / bf16) if alg else None,
                                    "executed_tflops": 3.0 * alg if alg else None,
                                    "executed_frac": (3.0 * alg / bf16) if alg else None,
                                    "peak_source": "MEASURED_PEAKS.json bf16_tflops (FP16 and BF16 run at the same "
                                                   "dense rate); of measured",
                                    "note": "algorithmic = each multiply-add of the update once; executed = the "
                                            "three MMAs of the split (hi*hi, hi*lo, lo*hi)"},
                         "tc_kind": {0: "none", 1: "tf32 split", 2: "fp16 split"}.get(int(st_m.get("tc_kind", 0))),
                         "launches_per_step": mixed["schur_launches"],
                         "flops_per_launch": mixed["schur_flops"] / nl,
                         "phase_ms_mixed": mixed.get("phase_ms"), "phase_ms_fp64": fp64.get("phase_ms"),
                         "fp64_kernel": {"kernel": "k_schur_dmma (outer update of large fronts, FP64 tensor-core "
                                                   "path: mma.sync m8n8k4 f64, 128x64 half tiles, 2 CTAs/SM)",
                                         "achieved": ach64, "peak": peaks["fp64_tflops"], "unit": "TFLOP/s",
                                         "peak_source": "cuBLAS DGEMM 8192^3 measured here (MEASURED_PEAKS.json "
                                                        "has no FP64 figure)",
                                         "frac": (ach64 / peaks["fp64_tflops"]) if ach64 else None}},
            "peaks_measured": peaks,
            "peaks_file": {k: filepk.get(k) for k in ("hbm_gbs", "bf16_tflops", "bf16_tflops_sustained")},
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(round(mixed["factor_launches"] + mixed["solve_launches"])) * args.steps,
            "gpu_launches_note": "kernels of the mixed path in the timed region (factor + refined solve, all steps); "
                                 "the factor and the solve sweeps run as replayed CUDA graphs",
            **extras,
        }
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# reference arm: the reference's CPU algorithm (oracle port) on the host cores
# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    """The K timed steps together run one whole rustyfem_factor + rustyfem_solve of the
    cube by the oracle with all host threads: step 0 the analysis, then the numeric
    factorization up the elimination tree by depth (the subtrees below a depth first,
    then one depth per step, oracle/refcpu.cpp oref_staged_*), the last step the solve.
    value = the numeric factorization + solve (as our arm's value), e2e = all of it."""
    if rank != 0:
        return
    from oracle import refcpu
    from rustyfem_b200 import workloads as W

    n = args.n
    refcpu.set_threads(0)
    cores = refcpu.threads()
    warm = W.hex8_cube(8).full()
    for _ in range(args.warmup):
        hw, _, _ = refcpu.factor(warm)
        hw.solve(warm.rhs)
        hw.free()
    model = W.hex8_cube(n).full()
    K = max(1, args.steps)
    # at most 4 factor parts (the subtrees below depth 3, then depths 2, 1, 0): each part
    # ends with a join that the plain recursion does not have, and more of them slow the
    # CPU factorization down measurably (about 15 % with 18 parts on the 40³ cube)
    nparts = min(max(1, K - 2), REF_FACTOR_PARTS)
    stages = ["analysis"] + [f"factor part {p}" for p in range(nparts)] + ["solve"]
    # stages spread over the steps, the analysis in the first and the solve in the last;
    # with more steps than stages some steps are empty
    ns = len(stages)
    step_of = [0] * ns if K == 1 else [int(round(i * (K - 1) / (ns - 1))) for i in range(ns)]
    step_s = [0.0] * K
    kind_s = {"analysis": 0.0, "factor": 0.0, "solve": 0.0}
    S = None
    h = None
    x = None
    for st, (name, k) in enumerate(zip(stages, step_of)):
        t0 = time.perf_counter()
        if name == "analysis":
            S = refcpu.StagedFactor(model, nparts)
        elif name == "solve":
            h, err = S.finish()
            if h is None:
                raise RuntimeError(f"oracle factorization failed at DOF {err}")
            x = h.solve(model.rhs)
        else:
            if not S.part(st - 1):
                raise RuntimeError("oracle factorization failed")
        dt = time.perf_counter() - t0
        step_s[k] += dt
        kind_s[name.split()[0]] += dt
    work, _ = h.info()
    nfronts = len(h.fronts())
    h.free()
    del x
    value = kind_s["factor"] + kind_s["solve"]
    total = sum(step_s)
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total / K * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: 60^3 C3D8 unit cube, steel E=210e9 nu=0.3, x=0 clamped, fz=-1000 N on x=1",
        "config": workload_config(n, model, work, nfronts),
        "parallelism": f"host threads x{cores}",
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port",
                         "sample": f"the whole workload, measured once: the {K} timed steps together run one "
                                   f"rustyfem_factor + rustyfem_solve of the hex8 {n}^3 cube (FP64, {cores} host "
                                   "threads); value = numeric factorization + solve"},
        "e2e": {"value": total, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timing": {"step_s": step_s, "stages_per_step": [[nm for nm, k in zip(stages, step_of) if k == i]
                                                          for i in range(K)],
                   "plain_factor_note": "the factor parts go up the tree by depth with a join after each; with "
                                        f"{nparts} parts the CPU factorization takes about as long as in one piece",
                   "analysis_s": kind_s["analysis"], "factor_s": kind_s["factor"], "solve_s": kind_s["solve"],
                   "note": "ms_per_step = the timed total / steps (the steps are slices of one run, of unequal "
                           "length, some empty when there are more steps than stages); value = factor + solve; e2e "
                           "= analysis + factor + solve (what one rustyfem_factor + rustyfem_solve call pair "
                           "costs)"},
        "note": "the reference is Rust (no cargo in this image): its multifrontal solver is timed through the "
                "C++ restatement in oracle/ with all host threads; the factorization is split into parts by "
                "elimination-tree depth (bit-identical factor, each subtree with the threads the plain recursion "
                "gives it)",
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.profile_only:
        run_profile_case(args)
        return
    if args.workload == "hex20":
        run_hex20(args)
        return
    if args.workload == "assembly":
        print(json.dumps(measure_assembly(args.n, not args.no_oracle)), flush=True)
        return
    if args.workload == "unsym":
        print(json.dumps(measure_unsym(args.n, not args.no_oracle)), flush=True)
        return
    if args.workload == "plates":
        run_plates(args)
        return
    if args.workload == "indef":
        print(json.dumps(measure_indef(30 if args.n == WORKLOAD_N else args.n, not args.no_oracle)), flush=True)
        return
    run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
