"""The bench's reference arm (the CPU implementation of the path, timed on the
host cores) runs without a GPU and prints one JSON line with the contract's
keys: the same metric and unit as the GPU arm, `impl: reference`, a
`cpu_baseline` describing the run and an `e2e` object without copies."""
import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    gpu_metric = re.search(r'^METRIC = "(.*)"$', open(os.path.join(ROOT, "bench.py")).read(), re.M).group(1)
    assert d["metric"] == gpu_metric
    assert d["unit"] == "Mops/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["warmup"] >= 3
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # the same-box comparison with the reference's GPU build needs a GPU
    assert "reference_gpu" in d
