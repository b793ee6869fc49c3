"""The reference arm of bench.py on the host (no GPU): one JSON line with the contract's
keys, timed on the oracle port, with the same workload description as our arm."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--n", "8"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "s" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["ms_per_step"] == line["value"] * 1e3
    assert line["steps"] == 1 and line["warmup"] == 0 and line["n_gpus"] == 1
    cfg = line["config"]
    assert cfg["workload"].startswith("hex8 8^3 elasticity (n=") and cfg["leaf"] == 16 and cfg["nrhs"] == 1
    assert cfg["flops"] > 0 and cfg["nfronts"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
