"""The reference arm of bench.py (CPU only): `--impl reference` prints one JSON
line with the contract's keys, on the same metric and unit as the GPU arm, timed
on the reference's own CPU code from oracle/_ref; under torchrun only rank 0
prints. Run on a small sample graph so the suite stays fast."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "impl"}


def _run(env_extra, *args):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


@pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built (reference CPU path)")
def test_reference_arm_prints_one_contract_line():
    lines = _run({}, "--impl", "reference", "--steps", "1", "--warmup", "0", "--cpu-sample-scale", "12")
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert "unavailable" not in d, d
    assert KEYS <= set(d), KEYS - set(d)
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "GTEPS"
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["scale"] == 12
    assert set(d["per_algorithm"]) == {"bfs", "cc", "pagerank"}


def test_reference_arm_is_silent_on_other_ranks():
    assert _run({"RANK": "1", "WORLD_SIZE": "2"}, "--impl", "reference", "--steps", "1", "--warmup", "0",
                "--cpu-sample-scale", "12") == []


@pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built (reference CPU path)")
def test_gpu_arm_cpu_baseline_runs_on_the_host():
    import bench
    cb = bench.reference_cpu_baseline(12)
    assert "unavailable" not in cb, cb
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["unit"] == "GTEPS" and cb["value"] > 0
    assert set(cb["per_algorithm"]) == {"bfs", "cc", "pagerank"}
    assert {"sssp_dijkstra", "ppr_vector", "pagerank_adjoint"} <= set(cb["restatements"])
