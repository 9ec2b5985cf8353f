"""Failure paths, injected on the host (nothing here faults, traps or hangs the
device): device allocations that fail from the k-th one on must surface as
MG_ERR_OOM from whichever call was running and leave the library usable; a
persistent-kernel grid barrier that cannot complete (test hook: one arrival more
than there are blocks, a short poll budget) must come back as MG_ERR_TIMEOUT with
the device still usable; repeated runs are bit-identical."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _workload(h):
    """Every allocating entry point once; returns the results."""
    out = {}
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        out["bfs"] = g.bfs([0])[0]
        out["sssp"] = g.sssp([0])[0]
        out["cc"] = g.cc()[0]
        out["pr"] = g.pagerank(mode="normalized", gather="cached")[0]
        out["prr"] = g.pagerank()[0]
        out["batch"] = g.bfs_batch([0, 5, 9])[0]
    return out


def test_allocation_failures_surface_as_oom_and_leave_the_library_usable():
    lib = L.load()
    h = mg.gen_rmat(12, 8, 31, weights="int", p0=1, p1=50)
    clean = _workload(h)
    seen_oom = 0
    try:
        for k in range(1, 40):
            assert lib.mg_debug_fail_alloc(k) == L.MG_OK
            try:
                _workload(h)
            except mg.MapGraphError as e:
                assert e.status == L.MG_ERR_OOM, str(e)
                seen_oom += 1
            finally:
                lib.mg_debug_fail_alloc(0)
            again = _workload(h)  # disarmed: everything works and agrees
            for key, v in clean.items():
                if key in ("pr",):
                    assert np.abs(again[key] - v).sum() <= 1e-6
                else:
                    np.testing.assert_array_equal(again[key], v)
    finally:
        lib.mg_debug_fail_alloc(0)
    assert seen_oom >= 10
    np.testing.assert_array_equal(clean["bfs"], oracle.bfs(h.row_offsets, h.col_idx, [0]))


def test_barrier_that_cannot_complete_times_out_and_the_device_stays_usable():
    lib = L.load()
    h = mg.gen_lattice(300, 200, 0.0, 5)  # small frontiers: the persistent BFS kernel runs
    ref = oracle.bfs(h.row_offsets, h.col_idx, [0])
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        try:
            assert lib.mg_debug_barrier_skew(1, 1 << 12) == L.MG_OK
            with pytest.raises(mg.MapGraphError) as ei:
                g.bfs([0])
            assert ei.value.status == L.MG_ERR_TIMEOUT
        finally:
            lib.mg_debug_barrier_skew(0, 1)
        d, st = g.bfs([0])
        np.testing.assert_array_equal(d, ref)
        assert st["iterations"] == ref.max() + 1
    assert lib.mg_debug_barrier_skew(-1, 5) == L.MG_ERR_ARG
    assert lib.mg_debug_fail_alloc(-3) == L.MG_ERR_ARG


def test_repeated_runs_are_bit_identical():
    # Integer outputs are bit-identical run to run. PageRank rows are too, except
    # that its FP64 residual and dangling-mass sums add per-CTA partials whose
    # row sets follow the dynamic schedule, so a value can move by one ulp.
    h = mg.gen_rmat(14, 16, 2, symmetrize=True, weights="int", p0=1, p1=255)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        runs = [(g.bfs([3])[0], g.sssp([3])[0], g.cc()[0], g.pagerank(mode="normalized")[0],
                 g.pagerank(mode="normalized", gather="cached")[0]) for _ in range(2)]
    for a, b in zip(runs[0][:3], runs[1][:3]):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(runs[0][3:], runs[1][3:]):
        assert np.abs(a - b).sum() <= 1e-9


def test_asynchronous_upload_overlaps_and_validates_on_first_use():
    h = mg.gen_rmat(13, 16, 77, symmetrize=True)
    ref = oracle.bfs(h.row_offsets, h.col_idx, [3])
    g1 = mg.Graph(h.row_offsets, h.col_idx, symmetric=True, async_upload=True)
    g2 = mg.Graph(h.row_offsets, h.col_idx, symmetric=True, async_upload=True)  # both uploads in flight
    try:
        np.testing.assert_array_equal(g1.bfs([3])[0], ref)
        g2.sync()
        np.testing.assert_array_equal(g2.bfs([3])[0], ref)
    finally:
        g1.close()
        g2.close()
    bad = h.col_idx.copy()
    bad[7] = h.n + 5
    g3 = mg.Graph(h.row_offsets, bad, symmetric=True, async_upload=True)  # accepted: checked on first use
    try:
        with pytest.raises(mg.MapGraphError) as ei:
            g3.bfs([0])
        assert ei.value.status == L.MG_ERR_ARG
        with pytest.raises(mg.MapGraphError):
            g3.sync()
    finally:
        g3.close()
    # a graph that needs a CSC uploads synchronously whatever the flag
    with pytest.raises(mg.MapGraphError):
        mg.Graph(h.row_offsets, bad, async_upload=True)
