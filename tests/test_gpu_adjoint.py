"""PageRank adjoint on the GPU (mg_pagerank_backward) against the FP64 CPU adjoint
and central finite differences of the FP64 forward solve.

Tolerance: gradient errors are measured norm-wise over the checked entries,
||g_gpu - g_ref|| / ||g_ref|| <= 1e-4."""
import concurrent.futures as cf

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = pytest.mark.gpu

REL = 1e-4


def _problem(scale, seed, weighted=True, teleport=False):
    h = mg.gen_rmat(scale, 16, seed, symmetrize=False, weights="lognormal" if weighted else None, p0=0, p1=1)
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(h.n)
    t = None
    if teleport:
        t = rng.random(h.n)
        t /= t.sum()
    a = h.weights_f32 if weighted else None
    x, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, a, 0.85, 1e-15, 5000, t)
    return h, a, w, t, x


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("weighted", [True, False])
@pytest.mark.parametrize("teleport", [False, True])
def test_adjoint_matches_fp64_adjoint(weighted, teleport):
    h, a, w, t, x = _problem(12, 5 + weighted + 2 * teleport, weighted, teleport)
    ga, gt, lam, _ = oracle.pr_adjoint(h.row_offsets, h.col_idx, a, x, w, teleport=t)
    with mg.Graph(h.row_offsets, h.col_idx, a) as g:
        gw, gtt, st = g.pagerank_backward(x.astype(np.float32), w.astype(np.float32),
                                          teleport=None if t is None else t.astype(np.float32),
                                          weighted=weighted, tol=1e-9, max_iter=400)
        assert _rel(gw, ga) <= REL and _rel(gtt, gt) <= REL
        for gather in ("tma",):
            gw2, gt2, _ = g.pagerank_backward(x.astype(np.float32), w.astype(np.float32),
                                              teleport=None if t is None else t.astype(np.float32),
                                              weighted=weighted, tol=1e-9, max_iter=400, gather=gather)
            assert _rel(gw2, ga) <= REL and _rel(gt2, gt) <= REL


def test_adjoint_finite_differences_1000_edges():
    """Forward and backward both on the GPU; central differences of L = w . x at
    1,000 seeded edges with h = 1e-3 |a_uv| in FP64 forward solves."""
    h, a, w, t, x64 = _problem(12, 17, True, False)
    with mg.Graph(h.row_offsets, h.col_idx, a) as g:
        x, st = g.pagerank(mode="normalized", weighted=True, tol=1e-9, max_iter=400)
        gw, gt, _ = g.pagerank_backward(x, w.astype(np.float32), weighted=True, tol=1e-9, max_iter=400)
    rng = np.random.default_rng(99)
    edges = rng.choice(h.m, size=1000, replace=False)
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


def test_adjoint_device_arrays_and_determinism():
    torch = pytest.importorskip("torch")
    h, a, w, t, x = _problem(11, 3, True, False)
    with mg.Graph(h.row_offsets, h.col_idx, a) as g:
        xd = torch.from_numpy(x.astype(np.float32)).cuda()
        wd = torch.from_numpy(w.astype(np.float32)).cuda()
        ow = torch.empty(h.m, dtype=torch.float32, device="cuda")
        ot = torch.empty(h.n, dtype=torch.float32, device="cuda")
        g.pagerank_backward(xd, wd, weighted=True, out_weights=ow, out_teleport=ot, tol=1e-9, max_iter=400)
        gw, gt, _ = g.pagerank_backward(x.astype(np.float32), w.astype(np.float32), weighted=True, tol=1e-9,
                                        max_iter=400)
        assert np.abs(ow.cpu().numpy() - gw).max() <= 1e-6 * max(1.0, np.abs(gw).max())
        assert np.abs(ot.cpu().numpy() - gt).max() <= 1e-6 * max(1.0, np.abs(gt).max())


def test_adjoint_rejects_refcompat_mode():
    h, a, w, t, x = _problem(8, 1, True, False)
    with mg.Graph(h.row_offsets, h.col_idx, a) as g:
        with pytest.raises(mg.MapGraphError):
            g.pagerank_backward(x.astype(np.float32), w.astype(np.float32), mode="refcompat")
