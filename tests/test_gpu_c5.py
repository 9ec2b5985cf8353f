"""The PageRank forward + adjoint workload at its stated size: R-MAT scale 24,
edge factor 16, directed (268 M edges), lognormal(0, 1) edge weights normalised by
their row sums, alpha 0.85, L = w . x with w ~ N(0, 1).

- Forward (FP32, compensated, FP64 residual) against the FP64 oracle at the same
  iteration count: L1 <= 1e-6.
- Backward (mg_pagerank_backward) against the FP64 CPU adjoint on the full graph,
  both from the same ranks: ||g_gpu - g_fp64|| / ||g_fp64|| <= 1e-4 for the edge
  and the teleport gradients.
- Central finite differences of the FP64 forward solve on 1,000 seeded edges
  (h = 1e-3 |a_uv|) at scale 16: 2,000 FP64 solves at scale 24 would take hours on
  the host, so the differences run at the largest scale that fits a test.

The forward normalised mode restates the reference's PageRank program
(Algorithms/PageRank/PageRank.h:233-283) with a row-normalised weighted P."""
import concurrent.futures as cf

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6
REL = 1e-4
SEED = 20140601


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def c5():
    h = mg.gen_rmat(24, 16, SEED + 12, symmetrize=False, weights="lognormal", p0=0, p1=1)
    w = np.random.default_rng(SEED + 13).standard_normal(h.n)
    return h, w


def test_c5_forward_matches_fp64(c5):
    h, _ = c5
    assert h.n == 1 << 24 and h.m > 250_000_000
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_f32) as g:
        for gather in ("binned", "segmented"):
            x, st = g.pagerank(mode="normalized", weighted=True, tol=1e-6, max_iter=200, gather=gather)
            xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, h.weights_f32, 0.85, 0.0, st["iterations"])
            err = float(np.abs(x.astype(np.float64) - xr).sum())
            assert err <= L1_TOL, (gather, err)


def test_c5_adjoint_matches_fp64_adjoint_on_the_full_graph(c5):
    h, w = c5
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_f32) as g:
        x, st = g.pagerank(mode="normalized", weighted=True, tol=1e-6, max_iter=200)
        gw, gt, stb = g.pagerank_backward(x, w.astype(np.float32), weighted=True, tol=1e-7, max_iter=400)
    # the oracle stops on the absolute L1 change of lambda: 1e-9 relative to ||w||_1
    ga, gtr, _, _ = oracle.pr_adjoint(h.row_offsets, h.col_idx, h.weights_f32, x.astype(np.float64), w,
                                      tol=1e-9 * float(np.abs(w).sum()), max_iter=1000)
    assert _rel(gw, ga) <= REL
    assert _rel(gt, gtr) <= REL


def test_c5_finite_differences_1000_edges_s16():
    h = mg.gen_rmat(16, 16, SEED + 14, symmetrize=False, weights="lognormal", p0=0, p1=1)
    a = h.weights_f32
    w = np.random.default_rng(SEED + 15).standard_normal(h.n)
    x64, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, a, 0.85, 1e-15, 5000)
    with mg.Graph(h.row_offsets, h.col_idx, a) as g:
        x, st = g.pagerank(mode="normalized", weighted=True, tol=1e-9, max_iter=400)
        gw, _, _ = g.pagerank_backward(x, w.astype(np.float32), weighted=True, tol=1e-9, max_iter=400)
    edges = np.random.default_rng(SEED + 16).choice(h.m, size=1000, replace=False)
    a64 = a.astype(np.float64)

    def fd(e):
        step = 1e-3 * a64[e]
        ap, am = a64.copy(), a64.copy()
        ap[e] += step
        am[e] -= step
        ap32, am32 = ap.astype(np.float32), am.astype(np.float32)
        lp = oracle.pr_loss(h.row_offsets, h.col_idx, ap32, w, x64, tol=1e-15, max_iter=5000)
        lm = oracle.pr_loss(h.row_offsets, h.col_idx, am32, w, x64, tol=1e-15, max_iter=5000)
        return (lp - lm) / (float(ap32[e]) - float(am32[e]))

    with cf.ThreadPoolExecutor(max_workers=16) as ex:
        ref = np.array(list(ex.map(fd, edges)))
    assert _rel(gw[edges], ref) <= REL
