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
    lines = _run({}, "--impl", "reference", "--steps", "1", "--warmup", "0", "--ref-scale", "12")
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
                "--ref-scale", "12") == []


@pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built (reference CPU path)")
def test_reference_arm_divides_the_passes_among_processes():
    """Three timed passes and two warm-up passes over the processes: every timed
    pass counted once (one BFS source each), the graph of the GPU arm's scale."""
    lines = _run({}, "--impl", "reference", "--steps", "3", "--warmup", "2", "--ref-scale", "11")
    d = json.loads(lines[0])
    assert "unavailable" not in d, d
    assert d["config"]["scale"] == 11 and d["steps"] == 3
    assert 1 <= d["cpu_baseline"]["cores"] <= 3
    import bench
    h = bench.cpu_sample_graph(11)
    assert d["value"] > 0 and h.m == d["config"]["m"]
    # CC counts m edges per pass: exactly three passes were timed
    cc = d["per_algorithm"]["cc"]
    assert abs(cc["gteps_per_core"] * cc["core_seconds"] * 1e9 - 3 * h.m) < 1e-3 * h.m


def test_pagerank_fp64_check_measures_the_error():
    """The CPU baseline leg's PageRank check: an exact FP64 result has no error,
    a perturbed one shows its L1 distance."""
    import numpy as np
    import bench
    h = bench.cpu_sample_graph(10)
    x, it, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, bench.ALPHA, 0.0, 12)
    chk = bench.pagerank_fp64_check(h, x.astype(np.float32), 12, fixed_point=True)
    assert chk["l1_vs_fp64"] < 1e-6 and chk["iterations"] == 12
    assert chk["fixed_point_iterations"] > 12 and chk["l1_vs_fp64_fixed_point"] > chk["l1_vs_fp64"]
    y = x.copy()
    y[0] += 1e-3
    assert abs(bench.pagerank_fp64_check(h, y, 12, fixed_point=False)["l1_vs_fp64"] - 1e-3) < 1e-9


@pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built (reference CPU path)")
def test_gpu_arm_cpu_baseline_runs_on_the_host():
    import bench
    cb = bench.reference_cpu_baseline(12)
    assert "unavailable" not in cb, cb
    assert cb["kind"] == "reference" and cb["cores"] == 1 and cb["unit"] == "GTEPS" and cb["value"] > 0
    assert set(cb["per_algorithm"]) == {"bfs", "cc", "pagerank"}
    assert {"sssp_dijkstra", "ppr_vector", "pagerank_adjoint"} <= set(cb["restatements"])
