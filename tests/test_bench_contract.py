"""The bench line's contract, checked on the arm that needs no GPU: `bench.py --impl reference`
times the reference's own CPU implementation (oracle/_ref, or the oracle port where the reference
library was not built) and prints one JSON line with the contract's keys."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "2", "--warmup", "1", "--cpu-seconds", "0.5"],
                       capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    b = json.loads(lines[0])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in b, key
    assert b["impl"] == "reference" and b["metric"] == "distance-evals/s"
    assert b["steps"] == 2 and b["warmup"] == 1 and b["higher_is_better"] is True
    assert b["value"] > 0 and b["ms_per_step"] > 0
    assert b["config"]["workload"].startswith("plain sgsknn float32")
    cb = b["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == b["value"]
    assert "2 timed calls" in cb["sample"]
    assert b["e2e"] == {"value": b["value"], "unit": b["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
