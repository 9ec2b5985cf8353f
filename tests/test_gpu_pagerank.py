"""PageRank on the GPU through the C ABI.

Reference-compatible mode: against the reference's CPUPR with the reference's own
check (relative L2 < tol = 0.1, Algorithms/PageRank/PageRank.cu:315-327) and
against the FP64 replay of the engine schedule. Normalised / personalised mode:
L1 <= 1e-6 against the FP64 oracle run for the same number of iterations."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6  # FP32 engine vs FP64 oracle, same iteration schedule
# Repeated runs agree to within 1e-9 L1, not bit for bit: the FP64 residual and
# dangling-mass sums add per-CTA partials whose rows follow the dynamic work
# schedule, so an element can move by one ulp.


def _fixture_graph(d):
    return mg.Graph(np.array(d["row_offsets"], dtype=np.int32), np.array(d["col_idx"], dtype=np.int32),
                    np.array(d["values"], dtype=np.float32))


@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_refcompat_fixtures(mtx_fixtures, name, use_graph):
    d = mtx_fixtures[name]
    ro, ci = np.array(d["row_offsets"]), np.array(d["col_idx"])
    with _fixture_graph(d) as g:
        x, st = g.pagerank(mode="refcompat", use_graph=use_graph)
    ref = np.array(d["cpupr"])
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 0.1
    x64, it = oracle.pr_refcompat(ro, ci, 1)
    assert st["iterations"] == it
    assert np.abs(x - x64).max() < 1e-5


def test_refcompat_golden_and_undirected(synthetic_golden):
    from golden.make_golden import er_graph, rmat_graph
    for key, h in (("er", er_graph()), ("rmat", rmat_graph())):
        with mg.Graph(h.row_offsets, h.col_idx) as g:
            x, st = g.pagerank(mode="refcompat")
            ref = synthetic_golden[key + "_pr"].astype(np.float64)
            assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 0.1
            x64, it = oracle.pr_refcompat(h.row_offsets, h.col_idx, 1)
            assert st["iterations"] == it
            assert np.abs(x - x64).max() < 1e-4
            xu, stu = g.pagerank(mode="refcompat", directed=0)
            xu64, itu = oracle.pr_refcompat(h.row_offsets, h.col_idx, 0)
            assert stu["iterations"] == itu
            assert np.abs(xu - xu64).max() < 1e-4


def _check_normalized(h, weights=None, teleport=None, symmetric=False, **kw):
    vals = None if weights is None else weights
    with mg.Graph(h.row_offsets, h.col_idx, vals, symmetric=symmetric) as g:
        x, st = g.pagerank(teleport=teleport, mode="normalized", weighted=weights is not None, **kw)
        it = st["iterations"]
        xr, it_r, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, weights, kw.get("alpha", 0.85), 0.0, it,
                                           None if teleport is None else teleport.astype(np.float64))
        assert it_r == it
        err = np.abs(x.astype(np.float64) - xr).sum()
        assert err <= L1_TOL, err
        return x, st, err


@pytest.mark.parametrize("scale,sym", [(10, True), (14, True), (14, False)])
def test_normalized_rmat(scale, sym):
    h = mg.gen_rmat(scale, 16, 3 + scale, symmetrize=sym)
    x, st, err = _check_normalized(h, symmetric=sym)
    assert st["iterations"] <= 50
    assert abs(x.astype(np.float64).sum() - 1.0) < 1e-5


def test_normalized_weighted_lognormal_directed():
    h = mg.gen_rmat(13, 16, 99, symmetrize=False, weights="lognormal", p0=0, p1=1)
    _check_normalized(h, weights=h.weights_f32)


def test_normalized_converges_on_tolerance():
    h = mg.gen_er(3000, 30000, 5)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        x, st = g.pagerank(mode="normalized", tol=1e-6, max_iter=500)
    assert st["residual"] < 1e-6 and st["iterations"] < 500
    xr, it, r = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 1e-6, 500)
    assert it == st["iterations"]
    assert np.abs(x - xr).sum() <= L1_TOL


def test_personalized_vectors_and_loop_modes():
    h = mg.gen_rmat(12, 8, 17, symmetrize=False)
    rng = np.random.default_rng(1)
    nvec = 5
    tele = np.zeros((nvec, h.n), dtype=np.float32)
    for k in range(nvec):
        sup = rng.choice(h.n, size=rng.integers(1, 33), replace=False)
        tele[k, sup] = 1.0 / sup.size
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        # nvec > 1 runs the batched solver: every vector for the same iterations.
        xs, st = g.pagerank(teleport=tele, nvec=nvec, mode="normalized")
        xs2, _ = g.pagerank(teleport=tele, nvec=nvec, mode="normalized", use_graph=False)
        assert np.abs(xs - xs2).sum() <= 1e-9 * nvec  # graph vs host-driven loop
        for k in range(nvec):
            xr, it, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"],
                                             tele[k].astype(np.float64))
            assert np.abs(xs[k] - xr).sum() <= L1_TOL
            x1, st1 = g.pagerank(teleport=tele[k], mode="normalized")
            xr, it, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st1["iterations"],
                                             tele[k].astype(np.float64))
            assert np.abs(x1 - xr).sum() <= L1_TOL


def test_pagerank_deterministic_and_hub_split():
    # a star: one row with far more edges than a tile holds, split over many tiles
    n = 20000
    ro = np.zeros(n + 1, dtype=np.int32)
    ro[1:] = n - 1  # vertex 0 -> all others
    ro[0] = 0
    ci = np.arange(1, n, dtype=np.int32)
    rows = np.concatenate([ro[:1], ro[1:]])
    # add the reverse edges: every leaf points back to 0
    src = np.concatenate([np.zeros(n - 1, dtype=np.int64), np.arange(1, n)])
    dst = np.concatenate([np.arange(1, n), np.zeros(n - 1, dtype=np.int64)])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    ro = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ro, src + 1, 1)
    ro = np.cumsum(ro).astype(np.int32)
    h = mg.HostCsr(ro, dst.astype(np.int32))
    x, st, err = _check_normalized(h, symmetric=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        a, _ = g.pagerank(mode="normalized")
        b, _ = g.pagerank(mode="normalized")
        assert np.abs(a - b).sum() <= 1e-9


def test_compensation_improves_accuracy():
    h = mg.gen_rmat(15, 16, 4, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        xc, st = g.pagerank(mode="normalized", compensated=True)
        xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
        assert np.abs(xc - xr).sum() <= L1_TOL


def test_api_pagerank_program(mtx_fixtures):
    d = mtx_fixtures["small"]
    ro, ci = np.array(d["row_offsets"], dtype=np.int32), np.array(d["col_idx"], dtype=np.int32)
    cfg = mg.Config(mg.pagerank)
    csr_problem = mg.CsrProblem(mg.pagerank, cfg)
    csr_problem.FromHostProblem(False, 7, 11, ci, ro, np.array(d["values"]), None, None, 1,
                                cfg.getParameter("directed"))
    mg.EnactorVertexCentric(csr_problem, mg.pagerank, cfg).EnactIterativeSearch(
        csr_problem, ro, cfg.getParameter("directed"), 7, None, cfg.getParameter("iter_num"),
        cfg.getParameter("threshold"))
    x = csr_problem.ExtractResults()
    ref = np.array(d["cpupr"])
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < cfg.getParameter("tol")


@pytest.mark.parametrize("gather", ["binned", "tma", "cached", "segmented"])
@pytest.mark.parametrize("weighted", [False, True])
def test_gather_kernels_agree_with_fp64(gather, weighted):
    h = mg.gen_rmat(14, 16, 61, symmetrize=False, weights="lognormal" if weighted else None, p0=0, p1=1)
    w = h.weights_f32 if weighted else None
    with mg.Graph(h.row_offsets, h.col_idx, w) as g:
        x, st = g.pagerank(mode="normalized", weighted=weighted, gather=gather)
        xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, w, 0.85, 0.0, st["iterations"])
        assert np.abs(x - xr).sum() <= L1_TOL
        x2, _ = g.pagerank(mode="normalized", weighted=weighted, gather=gather)
        assert np.abs(x - x2).sum() <= 1e-9


def test_gather_hub_chunks_binned():
    # one hub of 50k in-edges spans many chunks; leaves of degree 1
    n = 50001
    src = np.concatenate([np.arange(1, n), np.zeros(n - 1, dtype=np.int64)])
    dst = np.concatenate([np.zeros(n - 1, dtype=np.int64), np.arange(1, n)])
    order = np.lexsort((dst, src))
    ro = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ro, src[order] + 1, 1)
    h = mg.HostCsr(np.cumsum(ro).astype(np.int32), dst[order].astype(np.int32))
    for gather in ("binned", "tma", "cached", "segmented"):
        with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
            x, st = g.pagerank(mode="normalized", gather=gather)
        xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
        assert np.abs(x - xr).sum() <= L1_TOL


@pytest.mark.parametrize("weighted", [False, True])
def test_hub_column_cache_partial(weighted):
    # scale 17: more vertices with edges than the shared-memory column cache holds,
    # so gathers mix cached and uncached columns; results match the binned kernel
    # without the cache to rounding and the FP64 oracle within the usual bound.
    h = mg.gen_rmat(17, 16, 5, symmetrize=True, weights="lognormal" if weighted else None, p0=0, p1=1)
    assert (np.diff(h.row_offsets) > 0).sum() > 40000
    w = h.weights_f32 if weighted else None
    with mg.Graph(h.row_offsets, h.col_idx, w, symmetric=True) as g:
        x, st = g.pagerank(mode="normalized", weighted=weighted, gather="cached")
        xb, stb = g.pagerank(mode="normalized", weighted=weighted, gather="binned")
        xh, _ = g.pagerank(mode="normalized", weighted=weighted, gather="cached", use_graph=False)
    assert np.abs(x - xh).sum() <= 1e-9  # graph vs host-driven loop
    assert st["status_detail"] > 0 and stb["status_detail"] == 0  # cached columns reported
    assert st["iterations"] == stb["iterations"]
    xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, w, 0.85, 0.0, st["iterations"])
    assert np.abs(x - xr).sum() <= L1_TOL
    assert np.abs(x - xb).sum() <= L1_TOL


def test_gather_autotune_picks_and_keeps_a_variant():
    h = mg.gen_rmat(15, 16, 9, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        x, st = g.pagerank(mode="normalized", autotune=True)
        choice = st["status_detail"]  # cached columns of the chosen variant, 0 for none
        assert 0 <= choice <= h.n
        x2, st2 = g.pagerank(mode="normalized", autotune=True)  # tuned once per graph
        assert st2["status_detail"] == choice and np.abs(x - x2).sum() <= 1e-9
        xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
        assert np.abs(x - xr).sum() <= L1_TOL


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("sym", [True, False])
@pytest.mark.parametrize("hub_edges,block_cols", [(64, 4096), (16, 1024), (300, 8192), (1024, 40960)])
def test_segmented_gather_shapes(weighted, sym, hub_edges, block_cols):
    """The segmented gather over many column blocks: hub rows cut into fragments of
    every length class (and split at 1024 edges), phase 1 spread over the CTAs,
    the other rows through the column cache. Against the FP64 oracle at the same
    iteration count, and against the binned gather to rounding."""
    h = mg.gen_rmat(16, 16, 77, symmetrize=sym, weights="lognormal" if weighted else None, p0=0, p1=1)
    w = h.weights_f32 if weighted else None
    with mg.Graph(h.row_offsets, h.col_idx, w, symmetric=sym) as g:
        kw = dict(mode="normalized", weighted=weighted, gather="segmented", seg_hub_edges=hub_edges,
                  seg_block_cols=block_cols)
        x, st = g.pagerank(**kw)
        xh, sth = g.pagerank(use_graph=False, **kw)
        xb, stb = g.pagerank(mode="normalized", weighted=weighted, gather="binned")
    assert st["iterations"] == sth["iterations"] == stb["iterations"]
    assert np.abs(x - xh).sum() <= 1e-9
    xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, w, 0.85, 0.0, st["iterations"])
    assert np.abs(x - xr).sum() <= L1_TOL
    assert np.abs(x - xb).sum() <= L1_TOL


def test_segmented_gather_unsorted_rows_and_isolated_vertices():
    """Rows whose in-edges are not sorted by source (a symmetric CSR is gathered as
    given) still form one fragment per (row, block): the plan regroups each hub
    row's edges by block. Vertices without edges and a last block shorter than
    the rest are covered too."""
    rng = np.random.default_rng(5)
    h = mg.gen_rmat(15, 16, 13, symmetrize=True)
    ro, ci = h.row_offsets.copy(), h.col_idx.copy()
    for r in range(len(ro) - 1):  # shuffle every row
        rng.shuffle(ci[ro[r]:ro[r + 1]])
    with mg.Graph(ro, ci, symmetric=True) as g:
        x, st = g.pagerank(mode="normalized", gather="segmented", seg_hub_edges=32, seg_block_cols=3072)
    xr, _, _ = oracle.pr_normalized(ro, ci, None, 0.85, 0.0, st["iterations"])
    assert np.abs(x - xr).sum() <= L1_TOL


def test_segmented_gather_rejects_bad_shapes():
    h = mg.gen_rmat(12, 16, 3, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        with pytest.raises(mg.MapGraphError):
            g.pagerank(mode="normalized", gather="segmented", seg_block_cols=100)
        with pytest.raises(mg.MapGraphError):  # wider than a CTA's shared memory
            g.pagerank(mode="normalized", gather="segmented", seg_block_cols=1 << 20)
        x, st = g.pagerank(mode="normalized", gather="segmented")  # the graph is still usable
    xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
    assert np.abs(x - xr).sum() <= L1_TOL
