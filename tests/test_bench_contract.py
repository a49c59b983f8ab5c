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


def test_roofline_names_the_largest_class_with_a_byte_model():
    """bench._profile_roofline: the dominant kernel is the class with the most
    device time among those with algorithmic bytes; largest_classes lists the
    classes by time with their fraction of the peak where they have bytes."""
    import types
    import bench

    stats = [dict(name="scan_seeds", launches=4, items=10, bytes=0, ms=50.0),
             dict(name="radix_pass", launches=10, items=100, bytes=3_000_000_000, ms=40.0),
             dict(name="scan_rounds", launches=2, items=50, bytes=1_000_000_000, ms=45.0),
             dict(name="small", launches=1, items=1, bytes=10, ms=0.5)]

    class FakeCtx:
        def profile_reset(self):
            pass

        def profile(self, on):
            pass

        def profile_stats(self):
            return stats

    fake_torch = types.SimpleNamespace(cuda=types.SimpleNamespace(synchronize=lambda dev: None))
    roof, got = bench._profile_roofline(FakeCtx(), lambda: None, fake_torch, None)
    assert got is stats
    assert roof["kernel"] == "scan_rounds"  # 45 ms; scan_seeds has more time but no byte model
    assert abs(roof["achieved"] - 1e9 / 0.045 / 1e9) < 1e-6
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-12
    assert abs(roof["share_of_profiled_time"] - 45.0 / 135.5) < 1e-12
    names = [c["kernel"] for c in roof["largest_classes"]]
    assert names == ["scan_seeds", "scan_rounds", "radix_pass", "small"]
    assert roof["largest_classes"][0]["frac"] is None and roof["largest_classes"][2]["frac"] > 0
