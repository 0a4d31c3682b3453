"""The benchmark's reference arm runs the reference's CPU code only: the
trace workload's arm (bench.py --impl reference) builds the hierarchy with
the reference's own builder and traces with SoftwareGpu::Trace from
oracle/_ref, prints the contract's JSON line, and never loads the product
library or initialises CUDA."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

DRIVER = """
import runpy, sys, json
sys.argv = ["bench.py", "--impl", "reference", "--workload", "trace", "--steps", "1", "--warmup", "3"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
import torch
print(json.dumps({"product_loaded": "libre_b200" in maps, "oracle_ref_loaded": "libref_oracle" in maps,
                  "cuda_initialized": torch.cuda.is_initialized()}))
"""


def test_reference_arm_is_cpu_only(oracle):
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built")
    res = subprocess.run([sys.executable, "-c", DRIVER], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [json.loads(l) for l in res.stdout.splitlines() if l.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "Mrays/s"
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert probe == {"product_loaded": False, "oracle_ref_loaded": True, "cuda_initialized": False}
