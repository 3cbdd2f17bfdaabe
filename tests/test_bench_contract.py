"""The benchmark's reference arm runs on the host cores alone, so its JSON line
can be checked without a GPU: one timed step of config 1 through the
reference's own CPU step (oracle/_ref/ref_dump3d).  Skipped where oracle/_ref
was not built (the reference sources were absent when the package was built).
"""
import json
import os
import subprocess
import sys

import pytest

from oracle.oracle import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "ref_dump3d")),
                    reason="oracle/_ref not built (reference tree absent)")
def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "config1",
                          "--steps", "1", "--warmup", "1"],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "particle-steps/s" and d["unit"] == "particle-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 3  # the bench's warm-up floor
    assert d["ms_per_step"] > 0
    assert d["config"]["workload"] == "config1_dambreak_3d_dx10mm"
    # the same config object the GPU arm prints for the same arguments
    import argparse
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    from dem_mph_b200 import scenes
    args = argparse.Namespace(workload="config1", precision="fp32", no_bodies=False,
                              settle=bench.SETTLE_DEFAULT["config1"])
    assert d["config"] == json.loads(json.dumps(bench.workload_config(scenes.config1(seed=1234), args, 1)))
    assert "reference" in d["config"]["arms"] and "ours" in d["config"]["arms"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "sample" in cb
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
