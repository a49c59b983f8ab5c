"""The parts of bench.py that run without a GPU: the reference arm's JSON
line and the whole-build algorithmic byte model."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1", "--cpu-sample", str(1 << 20)],
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["unit"] == d["e2e"]["unit"] == "suffixes/s"
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert "workload" in d["config"] and "model" not in d["config"]


def test_algorithmic_build_bytes_model():
    import bench
    # (6w + 32) m + 28 n per level: a byte level of 1000 with 300 LMS, then a
    # u32 level of 300 with 90 LMS
    trace = [{"width": 1, "m": 1000, "n_lms": 300}, {"width": 4, "m": 300, "n_lms": 90}]
    assert bench.algorithmic_build_bytes(trace) == (6 + 32) * 1000 + 28 * 300 + (24 + 32) * 300 + 28 * 90
    assert bench.algorithmic_build_bytes(trace, 12 * 1000) == bench.algorithmic_build_bytes(trace) + 12000


@pytest.mark.parametrize("workload", ["genome1g", "batch4096", "zipf32", "iid8m", "derived", "short20k"])
def test_workload_configs_name_the_workload(workload):
    import bench
    sys.argv = ["bench.py", "--workload", workload]
    args = bench.parse()
    cfg = bench.workload_config(args)
    assert cfg["workload"] and "model" not in cfg
