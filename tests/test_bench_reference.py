"""The bench's reference arm on the CPU: `bench.py --impl reference` times the reference's CPU path
(its FP64 restatement under oracle/) on the host threads and prints one JSON line with the arm's
metric, `impl`, a `cpu_baseline` describing the run, the per-path work counters and an `e2e` that
moves no bytes. It needs no GPU, so it runs here as it runs on the GPU box."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_its_line():
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    run = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr[-2000:]
    lines = [l for l in run.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, run.stdout[-2000:]
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["unit"] == "paths/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "paths/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    work = line["per_path"]
    assert work["crossings"] > 0 and work["vertices"] > 0 and work["candidates"] > 0
    assert line["config"]["workload"].startswith("terrain square")
