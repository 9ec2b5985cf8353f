"""Per-level trace (mg_graph_trace, the reference's verbose per-iteration frontier
print): records written on the device by the level-end code agree with the
oracle's level structure and with the run's own counters."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["rmat", "lattice"])
def test_bfs_trace_matches_levels(kind):
    h = mg.gen_rmat(14, 16, 3, symmetrize=True) if kind == "rmat" else mg.gen_lattice(200, 100, 0.0, 1)
    ref = oracle.bfs(h.row_offsets, h.col_idx, [0])
    deg = np.diff(h.row_offsets)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        for mode in ("auto", "push"):
            _, st = g.bfs([0], direction=mode)
            tr = g.trace()
            assert len(tr) == st["iterations"] == ref.max() + 1
            counts = np.bincount(ref[ref >= 0])
            assert [r["frontier"] for r in tr] == counts.tolist()
            edges = [int(deg[ref == lvl].sum()) for lvl in range(len(counts))]
            assert [r["frontier_edges"] for r in tr] == edges
            assert sum(r["direction"] == "pull" for r in tr) == st["status_detail"]
            assert [r["level"] for r in tr] == list(range(len(tr)))
            assert all(r["ns"] >= 0 for r in tr[1:])  # level ends in order on the device clock


def test_sssp_and_pagerank_traces():
    h = mg.gen_rmat(13, 16, 8, symmetrize=True, weights="int", p0=1, p1=100)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        _, st = g.sssp([1])
        tr = g.trace()
        assert len(tr) == st["iterations"] and tr[0]["frontier"] == 1
        x, sp = g.pagerank(mode="normalized")
        tr = g.trace()
        assert len(tr) == sp["iterations"]
        assert all(r["frontier"] == h.n for r in tr)
        assert tr[-1]["value"] == pytest.approx(sp["residual"], rel=1e-12)
        assert all(a["value"] > b["value"] for a, b in zip(tr, tr[1:]))  # the L1 change falls
        g.cc()
        assert g.trace() == []  # CC records no levels
