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


def test_reference_arm_loads_no_product_library():
    """The reference arm's timing child builds its inputs from oracle/channel.py
    and times the reference's own build: it must map neither the product
    library nor its host emulator."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--cpu-child', 'reference:1:0']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "sys.stderr.write(open('/proc/self/maps').read())")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1])["steps"] == 1
    assert "libmpd_b200" not in r.stderr and "libmpd_emu" not in r.stderr
    assert "libmpd_ref.so" in r.stderr or "libmpd_oracle.so" in r.stderr


def test_oracle_channel_case_equals_the_package_case():
    """oracle/channel.py (no package) builds the same inputs as the config front end."""
    import numpy as np

    from oracle import bind, channel
    from tests import cases
    want = cases.channel_case(L=48, M=20).oracle_dict()
    for use_ref in ((True, False) if bind.ref_available() else (False,)):
        got = channel.channel_case(48, 20, use_reference=use_ref)
        for k in ("L", "M", "gamma", "beta", "H_z0", "dz", "dy", "r_0", "bc", "with_prev"):
            assert got[k] == want[k], k
        for k in ("rin", "rout", "drin", "drout", "phys"):
            assert np.array_equal(got[k], want[k]), k
