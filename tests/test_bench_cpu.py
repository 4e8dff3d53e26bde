"""bench.py without a GPU: the reference arm (the reference's CPU solver) prints
the fields the benchmark contract asks for and ranks other than 0 exit without
work; `--gpus N` launches its ranks itself and reports a split-room line."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(extra_env=None, *args):
    env = dict(os.environ, **(extra_env or {}))
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                          capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


def test_reference_arm_line():
    r = run_bench(None, "--steps", "1", "--warmup", "3", "--ref-seconds", "5")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == d["unit"] == "Gcell-updates/s"
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["config"]["grid"] == [512, 384, 256]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("reference", "port") and cb["cores"] >= 1
    assert "warm-up" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = run_bench({"RANK": "1", "WORLD_SIZE": "2"}, "--steps", "1", "--warmup", "3")
    assert r.returncode == 0
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_bench_launches_its_ranks_and_reports_a_split_run():
    """`bench.py --gpus 2` without a launcher starts two ranks itself; the
    plumbing check (gloo, a host stand-in for the step) prints rank 0's line
    with the split-room keys, and the other rank prints nothing."""
    import json
    import subprocess
    import sys
    res = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--plumbing-check",
                          "--steps", "3", "--warmup", "0"], capture_output=True, text=True, timeout=300,
                         env=dict(os.environ, MASTER_ADDR="127.0.0.1"))
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, res.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["scaling"] == "strong" and line["plumbing_check"]
    assert line["config"]["parallelism"] == "slab2"
    assert line["metric"] == "Gcell-updates/s" and line["steps"] == 3
