"""SSSP and CC on the GPU through the C ABI, bit-exact against the reference's
CPUSSSP / CPUCC (golden vectors) and the oracle."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200 import _lib as L
from conftest import ref_sssp_to_engine, INT_MAX

pytestmark = pytest.mark.gpu

LOOPS = [dict(), dict(use_graph=False)]


def _graph(d, symmetric=False):
    return mg.Graph(np.array(d["row_offsets"], dtype=np.int32), np.array(d["col_idx"], dtype=np.int32),
                    np.array(d["values"], dtype=np.int32), symmetric=symmetric)


@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
@pytest.mark.parametrize("loop", LOOPS)
def test_sssp_fixtures(mtx_fixtures, name, loop):
    d = mtx_fixtures[name]
    with _graph(d) as g:
        dist, _ = g.sssp([0], **loop)
        assert dist.tolist() == ref_sssp_to_engine(d["cpusssp_directed"]).tolist()
        if name == "chesapeake":
            dist, _ = g.sssp([0], directed=0, **loop)
            assert dist.tolist() == d["cpusssp_undirected"]


@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
def test_cc_fixtures(mtx_fixtures, name):
    d = mtx_fixtures[name]
    with _graph(d) as g:
        lab, st = g.cc()
        assert lab.tolist() == d["cpucc"]
        assert st["edges_traversed"] == len(d["col_idx"])


@pytest.mark.parametrize("loop", LOOPS)
def test_sssp_er_golden(synthetic_golden, loop):
    from golden.make_golden import er_graph
    G = synthetic_golden
    h = er_graph()
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        for i, s in enumerate(G["er_sources"]):
            dist, st = g.sssp([s], **loop)
            assert (dist == ref_sssp_to_engine(G["er_sssp"][i])).all()
            reached = dist != INT_MAX
            assert st["edges_traversed"] == int(np.diff(h.row_offsets)[reached].sum())


def test_sssp_cc_rmat_golden(synthetic_golden):
    from golden.make_golden import rmat_graph
    G = synthetic_golden
    h = rmat_graph()
    for sym in (False, True):
        with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=sym) as g:
            for i, s in enumerate(G["rmat_sources"]):
                dist, _ = g.sssp([s])
                assert (dist == ref_sssp_to_engine(G["rmat_sssp"][i])).all()
            assert (g.cc()[0] == G["rmat_cc"]).all()
    with mg.Graph(h.row_offsets, h.col_idx) as g:  # no weights: unit weights, distance = BFS depth
        bd = oracle.bfs(h.row_offsets, h.col_idx, [0])
        assert (g.sssp([0])[0] == np.where(bd < 0, INT_MAX, bd)).all()


@pytest.mark.parametrize("scale", [12, 16])
def test_sssp_rmat_vs_dijkstra(scale):
    h = mg.gen_rmat(scale, 16, 900 + scale, symmetrize=True, weights="int", p0=1, p1=255)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        for s in (0, 7, h.n - 1):
            ref = oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [s])
            for loop in LOOPS:
                assert (g.sssp([s], **loop)[0] == ref).all()


def test_sssp_directed_and_undirected_with_zero_weights():
    h = mg.gen_er(2000, 8000, 4, weights="int", p0=0, p1=5)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        for s in ([0], [10, 20, 10]):
            assert (g.sssp(s)[0] == oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, s, 1)).all()
            assert (g.sssp(s, directed=0)[0] == oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, s, 0)).all()


def test_sssp_lattice():
    h = mg.gen_lattice(120, 90, 0.001, 3, weights="int", p0=1, p1=1000)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        ref = oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [0])
        for loop in LOOPS:
            assert (g.sssp([0], **loop)[0] == ref).all()


def test_sssp_iter_num_and_errors():
    h = mg.gen_er(500, 3000, 8, weights="int", p0=1, p1=9)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        d1, st = g.sssp([0], iter_num=1)
        first = np.full(h.n, INT_MAX, dtype=np.int64)
        first[0] = 0
        b, e = h.row_offsets[0], h.row_offsets[1]
        for k in range(b, e):
            first[h.col_idx[k]] = min(first[h.col_idx[k]], h.weights_i32[k])
        assert (d1 == first).all() and st["iterations"] == 1
        with pytest.raises(mg.MapGraphError) as ex:
            g.sssp([500])
        assert ex.value.status == L.MG_ERR_ARG
    neg = h.weights_i32.copy()
    neg[3] = -1
    with mg.Graph(h.row_offsets, h.col_idx, neg) as g:
        with pytest.raises(mg.MapGraphError) as ex:
            g.sssp([0])
        assert ex.value.status == L.MG_ERR_ARG


@pytest.mark.parametrize("scale,sym", [(14, True), (17, True), (14, False)])
def test_cc_rmat_vs_oracle(scale, sym):
    h = mg.gen_rmat(scale, 8, 50 + scale, symmetrize=sym)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=sym) as g:
        lab, _ = g.cc()
        assert (lab == oracle.cc(h.row_offsets, h.col_idx)).all()
        assert (g.cc()[0] == lab).all()  # deterministic


def test_cc_many_components_and_lattice():
    # a ragged union of small graphs has one component per member at least
    parts = [mg.gen_er(50 + 7 * i, 60 + 5 * i, i) for i in range(20)]
    ro = [0]
    ci = []
    base = 0
    for p in parts:
        ro.extend((p.row_offsets[1:] + len(ci)).tolist())
        ci.extend((p.col_idx + base).tolist())
        base += p.n
    ro = np.array(ro, dtype=np.int32)
    ci = np.array(ci, dtype=np.int32)
    with mg.Graph(ro, ci) as g:
        assert (g.cc()[0] == oracle.cc(ro, ci)).all()
    h = mg.gen_lattice(300, 200, 0.0005, 2)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        assert (g.cc()[0] == 0).all()


def test_api_mirrors_reference_driver(mtx_fixtures):
    """The reference driver's call sequence (Algorithms/SSSP/sssp.cu:398-431)."""
    d = mtx_fixtures["small"]
    ro, ci, vals = (np.array(d[k], dtype=np.int32) for k in ("row_offsets", "col_idx", "values"))
    for prog, key in ((mg.bfs, "cpubfs_directed"), (mg.sssp, "cpusssp_directed"), (mg.cc, "cpucc")):
        cfg = mg.Config(prog)
        csr_problem = mg.CsrProblem(prog, cfg)
        csr_problem.FromHostProblem(False, 7, 11, ci, ro, vals, None, None, 1, 1)
        enactor = mg.EnactorVertexCentric(csr_problem, prog, cfg)
        srcs = None if prog is mg.cc else [0]
        enactor.EnactIterativeSearch(csr_problem, ro, 1, 1, srcs, cfg.getParameter("iter_num"),
                                     cfg.getParameter("threshold"))
        assert csr_problem.ExtractResults().tolist() == ref_sssp_to_engine(d[key]).tolist()


@pytest.mark.parametrize("delta", [-1, 0, 1, 7, 300, 1 << 24])
def test_sssp_near_far_bucket_widths(delta):
    # near-far (delta > 0) and plain Bellman-Ford (delta <= 0) reach the same
    # unique distances, in both loop drivers, on
    # weighted R-MAT, a directed ER graph read both ways and a lattice
    h = mg.gen_rmat(13, 16, 77, symmetrize=True, weights="int", p0=1, p1=255)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        for s in (0, 5, h.n - 1):
            ref = oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [s])
            for loop in LOOPS:
                d, st = g.sssp([s], delta=delta, **loop)
                assert (d == ref).all()
            dist_b, _ = g.sssp_batch([s, 1, 2], delta=delta)
            assert (dist_b[0] == ref).all()
    e = mg.gen_er(3000, 12000, 6, weights="int", p0=0, p1=40)
    with mg.Graph(e.row_offsets, e.col_idx, e.weights_i32) as g:
        for directed in (1, 0):
            d, _ = g.sssp([0, 9], delta=delta, directed=directed)
            assert (d == oracle.sssp(e.row_offsets, e.col_idx, e.weights_i32, [0, 9], directed)).all()
    lat = mg.gen_lattice(64, 80, 0.001, 2, weights="int", p0=1, p1=1000)
    with mg.Graph(lat.row_offsets, lat.col_idx, lat.weights_i32, symmetric=True) as g:
        d, st = g.sssp([0], delta=delta)
        assert (d == oracle.sssp(lat.row_offsets, lat.col_idx, lat.weights_i32, [0])).all()
        if delta > 0:
            assert st["status_detail"] == delta


def test_sssp_iteration_cap_keeps_reference_rounds():
    # with iter_num set the schedule is the reference's rounds even when a bucket
    # width is asked for
    h = mg.gen_er(500, 3000, 8, weights="int", p0=1, p1=9)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        a, _ = g.sssp([0], iter_num=2, delta=5)
        b, _ = g.sssp([0], iter_num=2, delta=-1)
        assert (a == b).all()
