"""bench.py --impl reference on the host (no GPU): the reference arm's JSON line, and under two
ranks only rank 0 runs and prints while rank 1 exits 0 without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [json.loads(t) for t in r.stdout.splitlines() if t.strip().startswith("{")]


def test_reference_line_keeps_the_contract():
    (line,) = run({})
    assert line["impl"] == "reference" and line["higher_is_better"] is True
    assert line["metric"] == "mDPD particle-steps/s (batched 256-box workload)" and line["unit"] == "particle-steps/s"
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 3 and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"].startswith("batched mDPD: 256 periodic boxes")


def test_second_rank_prints_nothing():
    assert run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
