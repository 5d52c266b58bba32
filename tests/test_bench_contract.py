"""bench.py's reference arm on CPU: one JSON line with the benchmark's
metric, unit and configuration, a cpu_baseline and an e2e object; under a
multi-rank launch only rank 0 prints, the other ranks exit 0 without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(env_extra, *args):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                          capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


def test_reference_arm_line():
    r = run_bench({}, "--impl", "reference", "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["unit"] == "paths/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 1
    assert d["config"]["paths"] == 65536 and d["config"]["paths_per_step"] >= 1
    assert d["scaling"] == "strong"
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("reference", "port")
    assert d["e2e"] == {"value": d["value"], "unit": "paths/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = run_bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"},
                  "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_sample_windows_span_the_range():
    sys.path.insert(0, ROOT)
    import bench
    w = bench.sample_windows(65536, 1024, 25)
    assert w[0] == 1 and w[-1] + 1024 - 1 == 65536
    assert all(b > a for a, b in zip(w, w[1:]))
    assert bench.sample_windows(65536, 1024, 1) == [1]
