"""The reference arm of bench.py (`--impl reference`): the reference's own
GAHHG kernels built for the CPU, timed on a bounded sample of the C1
workload, print one JSON line with the bench contract's keys.  Host only."""
import json
import os
import subprocess
import sys

from tests.conftest import REPO


def test_reference_arm_prints_its_line(oracle_ref):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, cwd=REPO, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    with open(os.path.join(REPO, "BASELINE.json")) as f:
        metric = json.load(f)["metric"]
    assert d["impl"] == "reference" and d["metric"] == metric
    assert d["unit"] == "Mpts/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert "C1" in d["config"]["workload"]
