"""bench.py's reference arm on the host cores: the JSON line contract.

The reference arm times the oracle port of the reference's CPU algorithm; it
runs without a GPU, so its line is checked here.  Rank 0 alone prints under a
multi-rank launch; other ranks exit without work.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    lines = _run({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "GB/s"
    assert d["config"]["workload"] == "regex" and d["steps"] == 1 and d["warmup"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("port", "reference") and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly():
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []


def test_boundary_guess_labels():
    # the regex record names how the walk chose its chunk starts: exact when
    # every speculative group starts exactly, else the tuner's choice
    sys.path.insert(0, str(ROOT))
    import bench
    info = {"n_groups": 3, "n_context_groups": 1, "exact_groups": 2}
    assert bench.boundary_guess(info, None).startswith("exact")
    info["exact_groups"] = 1
    assert bench.boundary_guess(info, {"proposer_used": 1}) == "learned proposer (top-1)"
    assert bench.boundary_guess(info, {"proposer_used": 0}).startswith("unanchored")
    assert bench.boundary_guess(dict(info, n_groups=1, n_context_groups=1, exact_groups=0), None).startswith("unanchored")
