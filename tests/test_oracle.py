"""The CPU oracle pinned to the reference: golden vectors recorded from the
reference's own CPUBFS/CPUSSSP/CPUCC/CPUPR, live comparisons when the reference
tree is present, and a finite-difference check of the FP64 PageRank adjoint."""
import hashlib
import os

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from conftest import ref_sssp_to_engine

pytestmark = pytest.mark.filterwarnings("ignore")

# Known-answer vectors of the three bundled graphs (reference CPU code, src = 0).
KAT = {
    "small": dict(bfs=[0, 1, 1, 1, 2, 2, 2], sssp=[0, 1, 4, 1, 2, 2, 2], cc=[0] * 7,
                  pr=[0.1500, 0.2470, 0.1925, 0.1925, 0.4145, 0.2864, 0.8276]),
    "trivialGraph": dict(bfs=[0, 1, 2, 3, 4], sssp=[0, 1, 2, 3, 4], cc=[0] * 5,
                         pr=[0.1500, 0.2775, 0.3859, 2.1589, 1.9851]),
}
CHESAPEAKE_UNDIRECTED_BFS = [0, 2, 2, 2, 2, 2, 1, 1, 2, 2, 1, 1, 1, 2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 2, 2, 2, 2, 2, 2, 2,
                             2, 2, 2, 1, 1, 2, 1, 2, 1]


def test_golden_matches_known_answers(mtx_fixtures):
    for name, kat in KAT.items():
        d = mtx_fixtures[name]
        assert d["cpubfs_directed"] == kat["bfs"]
        assert d["cpusssp_directed"] == kat["sssp"]
        assert d["cpucc"] == kat["cc"]
        assert np.allclose(d["cpupr"], kat["pr"], atol=5e-5)
    ch = mtx_fixtures["chesapeake"]
    assert ch["cpubfs_directed"] == [0] + [-1] * 38
    assert ch["cpusssp_directed"] == [0] + [100000000] * 38
    assert ch["cpubfs_undirected"] == CHESAPEAKE_UNDIRECTED_BFS
    assert ch["cpusssp_undirected"] == CHESAPEAKE_UNDIRECTED_BFS
    assert ch["n"] == 39 and len(ch["col_idx"]) == 170


@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
def test_restatement_matches_reference_on_fixtures(mtx_fixtures, name):
    d = mtx_fixtures[name]
    ro, ci, w = (np.array(d[k], dtype=np.int32) for k in ("row_offsets", "col_idx", "values"))
    csc = (np.array(d["col_offsets"], dtype=np.int32), np.array(d["row_idx"], dtype=np.int32), None)
    assert oracle.bfs(ro, ci, [0], 1).tolist() == d["cpubfs_directed"]
    assert oracle.sssp(ro, ci, w, [0], 1).tolist() == ref_sssp_to_engine(d["cpusssp_directed"]).tolist()
    assert oracle.cc(ro, ci).tolist() == d["cpucc"]
    if name == "chesapeake":
        assert oracle.bfs(ro, ci, [0], 0, csc=csc).tolist() == d["cpubfs_undirected"]
        assert oracle.sssp(ro, ci, w, [0], 0).tolist() == d["cpusssp_undirected"]
    # PageRank: the restatement follows the GPU engine's Jacobi delta-frontier
    # schedule, CPUPR is Gauss-Seidel; the reference's own check is relative L2 < tol = 0.1
    # (Algorithms/PageRank/PageRank.cu:315-327).
    x, _ = oracle.pr_refcompat(ro, ci, 1)
    ref = np.array(d["cpupr"])
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 0.1


def _digest(g):
    h = hashlib.sha256()
    for a in (g.row_offsets, g.col_idx, g.weights_i32):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_synthetic_golden(synthetic_golden):
    G = synthetic_golden
    from golden.make_golden import er_graph, rmat_graph
    for key, g in (("er", er_graph()), ("rmat", rmat_graph())):
        assert _digest(g) == bytes(G[key + "_digest"]).hex(), f"{key} generator output changed"
        for i, s in enumerate(G[key + "_sources"]):
            assert (oracle.bfs(g.row_offsets, g.col_idx, [s]) == G[key + "_bfs"][i]).all()
            assert (oracle.sssp(g.row_offsets, g.col_idx, g.weights_i32, [s]) ==
                    ref_sssp_to_engine(G[key + "_sssp"][i])).all()
        assert (oracle.cc(g.row_offsets, g.col_idx) == G[key + "_cc"]).all()
        x, _ = oracle.pr_refcompat(g.row_offsets, g.col_idx, 1)
        ref = G[key + "_pr"].astype(np.float64)
        assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 0.1


@pytest.mark.skipif(not oracle.have_ref(), reason="reference tree not present")
@pytest.mark.parametrize("seed", [1, 2, 3, 4, 5])
def test_restatement_matches_reference_random(seed):
    g = mg.gen_er(300, 1200, seed, weights="int", p0=0, p1=9)
    csc = oracle.csc_of(g.row_offsets, g.col_idx)
    R = oracle.Ref
    for s in (0, 7, 299):
        for directed in (1, 0):
            b, _ = R.bfs(g.row_offsets, g.col_idx, s, directed, csc)
            assert (b == oracle.bfs(g.row_offsets, g.col_idx, [s], directed, csc=csc)).all()
        d, _ = R.sssp(g.row_offsets, g.col_idx, g.weights_i32, s, 1, csc)
        assert (ref_sssp_to_engine(d) == oracle.sssp(g.row_offsets, g.col_idx, g.weights_i32, [s], 1)).all()
    c, _ = R.cc(g.row_offsets, g.col_idx, csc)
    assert (c == oracle.cc(g.row_offsets, g.col_idx)).all()


@pytest.mark.skipif(not oracle.have_ref(), reason="reference tree not present")
def test_market_reader_matches_reference_ingest():
    for name in ("small", "trivialGraph", "chesapeake"):
        path = os.path.join(oracle.REFERENCE_DIR, "smallRegressionGraphs", name + ".mtx")
        ro, ci, vals, co, ri = oracle.Ref.load_market(path)
        g = mg.read_market(path)
        assert (g.row_offsets == ro).all() and (g.col_idx == ci).all() and (g.weights_i32 == vals).all()
        co2, ri2, _ = mg.csr_to_csc(g)
        assert (co2 == co).all() and (ri2 == ri).all()


def test_multisource_bfs_is_min_over_sources():
    g = mg.gen_er(500, 1500, 11)
    srcs = [3, 77, 400]
    multi = oracle.bfs(g.row_offsets, g.col_idx, srcs)
    singles = np.stack([oracle.bfs(g.row_offsets, g.col_idx, [s]) for s in srcs]).astype(np.int64)
    singles[singles < 0] = 1 << 40
    best = singles.min(0)
    best[best == 1 << 40] = -1
    assert (multi == best).all()


def test_normalized_pagerank_fixed_point():
    g = mg.gen_rmat(8, 8, 3, symmetrize=False, weights="lognormal", p0=0, p1=1)
    x, it, r = oracle.pr_normalized(g.row_offsets, g.col_idx, g.weights_f32, tol=1e-13, max_iter=2000)
    assert r < 1e-13 and abs(x.sum() - 1.0) < 1e-10 and (x > 0).all()


def test_adjoint_matches_finite_differences():
    """The FP64 adjoint (the engine's backward formula) against central differences."""
    g = mg.gen_rmat(7, 6, 5, symmetrize=False, weights="lognormal", p0=0, p1=1)
    ro, ci, a = g.row_offsets, g.col_idx, g.weights_f32.astype(np.float32)
    n = g.n
    rng = np.random.default_rng(0)
    w = rng.standard_normal(n)
    t = rng.random(n)
    t /= t.sum()
    x, _, _ = oracle.pr_normalized(ro, ci, a, tol=1e-15, max_iter=5000, teleport=t)
    ga, gt, lam, _ = oracle.pr_adjoint(ro, ci, a, x, w, teleport=t)
    edges = rng.choice(g.m, size=40, replace=False)
    fd = []
    for e in edges:
        h = 1e-3 * float(a[e])
        ap, am = a.astype(np.float64).copy(), a.astype(np.float64).copy()
        ap[e] += h
        am[e] -= h
        lp = oracle.pr_loss(ro, ci, ap.astype(np.float32), w, x, teleport=t)
        lm = oracle.pr_loss(ro, ci, am.astype(np.float32), w, x, teleport=t)
        fd.append((lp - lm) / (np.float32(a[e] + h) - np.float32(a[e] - h)))
    fd = np.array(fd)
    assert np.linalg.norm(ga[edges] - fd) / np.linalg.norm(fd) < 1e-4
    # teleport gradient: dL/dt_i, perturbing t without renormalising
    for i in rng.choice(n, size=5, replace=False):
        h = 1e-4
        tp, tm = t.copy(), t.copy()
        tp[i] += h
        tm[i] -= h
        lp = oracle.pr_loss(ro, ci, a, w, x, teleport=tp)
        lm = oracle.pr_loss(ro, ci, a, w, x, teleport=tm)
        assert abs((lp - lm) / (2 * h) - gt[i]) <= 1e-4 * max(1.0, abs(gt[i]))


def test_bfs_pred_rule_on_a_path():
    # 0 -> 1 -> 2, 3 -> 2, 4 isolated: pred(1) = 0, pred(2) = 1 (3 is unreached),
    # the source takes its largest unreached in-neighbour (none here: -1)
    ro = np.array([0, 1, 2, 2, 3, 3], dtype=np.int32)
    ci = np.array([1, 2, 2], dtype=np.int32)
    depth = np.array([0, 1, 2, -1, -1], dtype=np.int32)
    assert oracle.bfs_pred(ro, ci, depth).tolist() == [-1, 0, 1, -1, -1]
