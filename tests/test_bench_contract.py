"""bench.py's output contract, on the CPU: the reference arm's JSON line (the
reference build, or the oracle port where it is absent, timed on the host
cores), and the GPU arm failing loudly without a device."""
import json
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _bench(*args, timeout=300):
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=timeout)


def test_reference_arm_line():
    r = _bench("--impl", "reference", "--steps", "2", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["metric"] == "cell-updates/s" and line["unit"] == "cell-updates/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] >= 1 and line["n_gpus"] == 1
    assert line["config"]["workload"].startswith("plain FP64 LF time step")
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "cell-updates/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_gpu_arm_fails_loudly_without_a_device(gpu_available):
    if gpu_available:
        pytest.skip("a GPU is present")
    r = _bench("--steps", "1", "--warmup", "1", timeout=600)
    assert r.returncode != 0
    assert not any(l.startswith("{") and '"value"' in l for l in r.stdout.splitlines())
