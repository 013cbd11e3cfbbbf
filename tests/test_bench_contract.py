"""The reference arm of bench.py on the host cores (no GPU): one JSON line with the keys
the benchmark contract names, on the same metric and workload as the device arm, and no
work on ranks other than 0."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True, cwd=ROOT,
                       env=e, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


def test_reference_arm_line():
    sys.path.insert(0, str(ROOT))
    import bench
    lines = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0")
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.SV_METRIC
    assert line["unit"] == "quotes/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["ms_per_step"] > 0
    assert (line["n_gpus"], line["steps"], line["warmup"]) == (1, 1, 0)
    assert line["vs_baseline"] is None and line["data"] == "synthetic"
    assert line["config"] == bench.sv_config("bf16x3", 1)
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == line["value"] and cb["unit"] == line["unit"]
    assert line["e2e"] == {"value": line["value"], "unit": "quotes/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_without_work():
    lines = run_bench("--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
                      env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert lines == []
