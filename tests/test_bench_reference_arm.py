"""The reference arm of bench.py on the host (no GPU): one JSON line with the contract's
keys, timed on the oracle port, with the same workload description as our arm. Its
timed steps are slices of one whole factor + solve of the cube: their sum is the
line's end-to-end time, and the factor + solve part of it is the line's value."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(steps, warmup, n):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps",
                          str(steps), "--warmup", str(warmup), "--n", str(n)], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("steps,warmup", [(1, 0), (2, 1), (5, 2), (20, 3)])
def test_reference_arm_prints_the_contract_line(steps, warmup):
    line = _run(steps, warmup, 8)
    assert line["impl"] == "reference"
    assert line["unit"] == "s" and line["higher_is_better"] is False
    assert line["steps"] == steps and line["warmup"] == warmup and line["n_gpus"] == 1
    tm = line["timing"]
    assert len(tm["step_s"]) == steps and all(t >= 0 for t in tm["step_s"])
    total = sum(tm["step_s"])
    # the timed region (steps x ms_per_step) is the one whole run, and e2e is its time
    assert abs(line["ms_per_step"] * steps / 1e3 - total) < 1e-9
    assert abs(line["e2e"]["value"] - total) < 1e-9
    assert abs(line["value"] - (tm["factor_s"] + tm["solve_s"])) < 1e-9 and 0 < line["value"] <= total
    stages = [s for per in tm["stages_per_step"] for s in per]
    assert stages[0] == "analysis" and stages[-1] == "solve"
    assert stages[1:-1] == [f"factor part {p}" for p in range(min(max(1, steps - 2), 4))]
    assert "analysis" in tm["stages_per_step"][0] and "solve" in tm["stages_per_step"][-1]
    cfg = line["config"]
    assert cfg["workload"].startswith("hex8 8^3 C3D8 elasticity (n=") and cfg["leaf"] == 16 and cfg["nrhs"] == 1
    assert cfg["flops"] > 0 and cfg["nfronts"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_same_config_as_our_arm():
    """Both arms describe the workload with bench.workload_config; the reference arm's
    flops and front count come from the oracle and equal the product's analysis."""
    sys.path.insert(0, ROOT)
    import bench
    from rustyfem_b200 import ffi, workloads as W

    line = _run(1, 0, 8)
    m = W.hex8_cube(8).full()
    sym = ffi.Symbolic(m.graph, 16)
    assert line["config"] == bench.workload_config(8, m, sym.work(), sym.nfronts)
