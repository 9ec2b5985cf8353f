"""The four programs on a seeded R-MAT scale-24 graph (16.8 M vertices, 536 M
directed edges after symmetrisation, weights U{1..255}): BFS depths and CC
labels bit-exact against the oracle, SSSP distances checked by the properties
that characterise exact shortest-path distances (every edge relaxed, every
reached vertex reached by a tight edge: together they force the true distances
for positive weights; Dijkstra at this size is too slow for a test), PageRank
within 1e-6 L1 of the FP64 oracle at the same iteration count. Minutes, not
seconds: most of it is the host-side generator and the FP64 oracle."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

INT_MAX = 2**31 - 1


def _check_shortest_paths(ro, ci, w, src, dist, chunk_rows=1 << 20):
    n = ro.size - 1
    assert dist[src] == 0
    d = dist.astype(np.int64)
    reached_v = dist != INT_MAX
    tight = np.zeros(n, dtype=bool)
    tight[src] = True
    for r0 in range(0, n, chunk_rows):
        r1 = min(n, r0 + chunk_rows)
        e0, e1 = int(ro[r0]), int(ro[r1])
        u = np.repeat(np.arange(r0, r1, dtype=np.int64), np.diff(ro[r0:r1 + 1]).astype(np.int64))
        v = ci[e0:e1]
        ok = reached_v[u]
        cand = d[u] + w[e0:e1]
        dv = d[v]
        # every edge out of a reached vertex is relaxed
        assert (dv[ok] <= cand[ok]).all()
        tight[v[ok & (dv == cand)]] = True
    # every reached vertex has a tight in-edge from a reached vertex
    assert tight[reached_v].all()


def test_four_programs_rmat_scale24():
    torch = pytest.importorskip("torch")
    h = mg.gen_rmat(24, 16, 20240601, symmetrize=True, weights="int", p0=1, p1=255)
    ro, ci, w = h.row_offsets, h.col_idx, h.weights_i32
    deg = np.diff(ro)
    src = int(np.argmax(deg > 0))
    with mg.Graph(ro, ci, w, symmetric=True) as g:
        depth, sb = g.bfs([src])
        dist, ss = g.sssp([src])
        label, _ = g.cc()
        x, sp = g.pagerank(mode="normalized", alpha=0.85, tol=1e-6, max_iter=50, autotune=True)
    np.testing.assert_array_equal(depth, oracle.bfs(ro, ci, [src]))
    assert sb["edges_traversed"] == int(deg[depth >= 0].sum())
    np.testing.assert_array_equal(label, oracle.cc(ro, ci))
    _check_shortest_paths(ro, ci, w, src, dist)
    np.testing.assert_array_equal(depth >= 0, dist != INT_MAX)
    xr, _, _ = oracle.pr_normalized(ro, ci, None, 0.85, 0.0, sp["iterations"])
    err = np.abs(x - xr).sum()
    print(f"R-MAT s24: PageRank L1 vs FP64 = {err:.3g} after {sp['iterations']} iterations")
    assert err <= 1e-6
