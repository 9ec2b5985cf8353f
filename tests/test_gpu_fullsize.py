"""Parity at the full sizes of the lattice and batched workloads (minutes, not
seconds; most of it is the host-side oracle):

- 4096 x 4096 lattice + 0.1% long-range pairs (16.8 M vertices, 67 M edges),
  weights U{1..1000}, from the corner: BFS depths and SSSP distances bit-exact
  against the oracle (BFS, Dijkstra);
- R-MAT scale 20 ef16 symmetrised, weights U{1..255}: a 64-source batched BFS and
  a 64-source batched SSSP bit-exact against the oracle on every source, and 256
  personalised PageRank vectors within 1e-6 L1 of the FP64 oracle on a sample of
  vectors."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

def test_lattice_4096_bfs_and_sssp():
    h = mg.gen_lattice(4096, 4096, 0.001, 20140601 + 3, weights="int", p0=1, p1=1000)
    ro, ci, w = h.row_offsets, h.col_idx, h.weights_i32
    with mg.Graph(ro, ci, w, symmetric=True) as g:
        depth, sb = g.bfs([0])
        dist, ss = g.sssp([0])
    ref = oracle.bfs(ro, ci, [0])
    np.testing.assert_array_equal(depth, ref)
    assert sb["iterations"] == ref.max() + 1
    np.testing.assert_array_equal(dist, oracle.sssp(ro, ci, w, [0]))


def test_batched_rmat_scale20_64_sources_and_256_vectors():
    torch = pytest.importorskip("torch")
    h = mg.gen_rmat(20, 16, 20140601 + 7, symmetrize=True, weights="int", p0=1, p1=255)
    ro, ci, w = h.row_offsets, h.col_idx, h.weights_i32
    srcs = mg.mixed_degree_sources(ro, 64, 20140601 + 8)
    tele = mg.sparse_teleports(h.n, 256, 20140601 + 9)
    with mg.Graph(ro, ci, w, symmetric=True) as g:
        depths, _ = g.bfs_batch(srcs)
        dists, _ = g.sssp_batch(srcs)
        xs, sp = g.pagerank(teleport=tele, nvec=256, mode="normalized", alpha=0.85, tol=1e-6, max_iter=50)
    for k, s in enumerate(srcs):
        np.testing.assert_array_equal(depths[k], oracle.bfs(ro, ci, [int(s)]))
        np.testing.assert_array_equal(dists[k], oracle.sssp(ro, ci, w, [int(s)]))
    for k in (0, 63, 128, 255):
        xr, it, _ = oracle.pr_normalized(ro, ci, None, 0.85, 0.0, sp["iterations"], tele[k].astype(np.float64))
        assert it == sp["iterations"]
        assert np.abs(xs[k].astype(np.float64) - xr).sum() <= 1e-6
