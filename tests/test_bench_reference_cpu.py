"""bench.py's reference arm (the reference's own build in oracle/_ref on the
host cores, else the oracle port) runs on the CPU; its JSON line keeps the
contract the GPU arm keeps: the same metric, unit and workload description,
the sample it timed, and an end-to-end entry with no host-device traffic.
The arm never loads the product library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "particle-steps/s" and d["higher_is_better"] is True
    assert (d["n_gpus"], d["steps"], d["warmup"]) == (1, 1, 1)
    assert d["config"] == bench.workload_config(1)
    assert d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_runs_the_reference_build_without_the_product_library():
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0'];"
            "runpy.run_path('bench.py', run_name='__main__');"
            "print('MAPPED', any('libldp' in l for l in open('/proc/self/maps')))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MAPPED False" in r.stdout
    d = json.loads(next(l for l in r.stdout.splitlines() if l.startswith("{")))
    if os.access(os.path.join(ROOT, "oracle", "_ref", "langevinDynamicsSingleBarrier"), os.X_OK):
        assert d["cpu_baseline"]["kind"] == "reference"
        assert "AVX-512" in d["cpu_baseline"]["sample"]
