"""bench.py's reference arm runs on the host alone: its JSON line carries the
keys the measurement contract names, the same metric and workload object as
the GPU arm, and a baseline description that matches the line."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _line(*extra):
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--doc-mib", "2", "--steps", "1",
                          "--warmup", "1", *extra], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    sys.path.insert(0, ROOT)
    import bench
    d = _line()
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "GB/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["n_gpus"] == 1 and d["steps"] >= 5
    assert d["dtype"] == "u8" and d["data"] == "synthetic" and d["vs_baseline"] is None
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == "GB/s"
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    cfg = d["config"]
    assert cfg["doc_bytes"] == 2 << 20 and len(cfg["input_sha256"]) == 64
    # the GPU arm names its workload with the same function, from the same generator
    import oracle
    doc = oracle.synth_json(2 << 20, bench.DEPTH, bench.SEED)
    assert cfg == bench._config(2 << 20, bench._sha256(doc))
