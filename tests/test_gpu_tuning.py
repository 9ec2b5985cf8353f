"""Traversal tuning (mg_graph_set_tuning): every setting of the thresholds and
launch shapes gives the same exact results, against the oracle; out-of-range
values are refused and change nothing."""
import numpy as np
import pytest

import mirrorofmapgraph_b200 as mg
import oracle
from mirrorofmapgraph_b200 import _lib as L

pytestmark = pytest.mark.gpu

SSSP_SETTINGS = [
    {},                                                  # defaults
    dict(sssp_heavy=1, sssp_heavy_small=1),              # every vertex cut into chunks
    dict(sssp_heavy=1 << 30, sssp_heavy_small=1 << 30),  # every vertex walked by its warp
    dict(sssp_heavy=64, sssp_heavy_small=8, sssp_chunk_cap=1),  # chunk list full: warps walk their vertices
    dict(sssp_heavy=32, sssp_chunk_cap=100),
    dict(sssp_ctas_per_sm=1),
    dict(sssp_ctas_per_sm=8, sssp_heavy=128),
    dict(sssp_batch_heavy=1),          # every batch item cut into chunks
    dict(sssp_batch_heavy=1 << 30),    # every batch item walked by its warp
    dict(sssp_batch_heavy=16, sssp_chunk_cap=3),
]


@pytest.fixture(scope="module")
def rmat13():
    h = mg.gen_rmat(13, 16, 606, symmetrize=True, weights="int", p0=1, p1=255)
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True)
    yield h, g
    g.close()


@pytest.mark.parametrize("setting", SSSP_SETTINGS, ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()) or "defaults")
def test_sssp_tuning_settings_are_exact(rmat13, setting):
    h, g = rmat13
    g.set_tuning(**{**mg.Graph.default_tuning(), **setting})
    try:
        srcs = [0, 17, h.n - 1]
        for s in srcs:
            ref = oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [s])
            for use_graph in (True, False):
                d, st = g.sssp([s], use_graph=use_graph)
                np.testing.assert_array_equal(d, ref)
                assert st["edges_traversed"] == int(np.diff(h.row_offsets)[ref < 2**31 - 1].sum())
            # near-far rounds through the same kernels
            np.testing.assert_array_equal(g.sssp([s], delta=40)[0], ref)
        db, _ = g.sssp_batch(srcs)
        for i, s in enumerate(srcs):
            np.testing.assert_array_equal(db[i], oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [s]))
    finally:
        g.set_tuning(**mg.Graph.default_tuning())


@pytest.mark.parametrize("setting", SSSP_SETTINGS[:4] + SSSP_SETTINGS[-3:],
                         ids=["defaults", "all-chunks", "all-walked", "cap-1", "batch-chunks", "batch-walked",
                              "batch-cap-3"])
def test_sssp_tuning_both_directions(setting):
    # directed graph read both ways: chunks of CSC edges carry the reverse flag
    h = mg.gen_rmat(12, 16, 31, symmetrize=False, weights="int", p0=0, p1=40)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        g.set_tuning(**{**g.tuning(), **setting})
        for directed in (1, 0):
            d, _ = g.sssp([0, 5], directed=directed)
            np.testing.assert_array_equal(d, oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [0, 5], directed))
            db, _ = g.sssp_batch([0, 5, 77], directed=directed)
            for i, s_ in enumerate([0, 5, 77]):
                np.testing.assert_array_equal(db[i], oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [s_],
                                                                 directed))


def test_tuning_ranges(rmat13):
    h, g = rmat13
    before = g.tuning()
    assert before == mg.Graph.default_tuning()
    for bad in (dict(sssp_heavy=0), dict(sssp_heavy_small=before["sssp_heavy"] + 1), dict(sssp_ctas_per_sm=9),
                dict(sssp_ctas_per_sm=0), dict(sssp_chunk_cap=-1), dict(sssp_batch_heavy=0)):
        with pytest.raises(mg.MapGraphError) as ex:
            g.set_tuning(**bad)
        assert ex.value.status == L.MG_ERR_ARG
        assert g.tuning() == before
    with pytest.raises(KeyError):
        g.set_tuning(no_such_field=1)


BFS_SETTINGS = [
    dict(bfs_cta_th=32, bfs_grid_th=64),                                 # CTA and grid bins take nearly all
    dict(bfs_cta_th=1 << 30, bfs_grid_th=1 << 30, bfs_defer_warp=0),     # warp and thread bins only
    dict(bfs_persist_max=0),                                             # no persistent levels
    dict(bfs_persist_max=1 << 30, bfs_persist_edges=1 << 30),            # every push level persistent
    dict(bfs_alpha=1, bfs_beta=1 << 20),
    dict(bfs_alpha=1 << 20, bfs_beta=1),
    dict(bfs_sparse_degree=1 << 20),                                     # AUTO stays top-down
    dict(bfs_ctas_per_sm=1),
    dict(bfs_ctas_per_sm=8),
    dict(bfs_tail_max=0),                                                # no single-CTA tail levels
    dict(bfs_tail_max=1 << 30, bfs_tail_edges=1 << 30, bfs_persist_max=0),  # every push level in one CTA
]


@pytest.mark.parametrize("setting", BFS_SETTINGS, ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()))
def test_bfs_tuning_settings_are_exact(rmat13, setting):
    h, g = rmat13
    g.set_tuning(**{**mg.Graph.default_tuning(), **setting})
    try:
        for s in (0, 99, h.n - 1):
            ref = oracle.bfs(h.row_offsets, h.col_idx, [s])
            for direction in ("auto", "push", "pull"):
                for use_graph in (True, False):
                    d, st = g.bfs([s], direction=direction, use_graph=use_graph)
                    np.testing.assert_array_equal(d, ref)
                    assert st["edges_traversed"] == int(np.diff(h.row_offsets)[ref >= 0].sum())
    finally:
        g.set_tuning(**mg.Graph.default_tuning())


def test_bfs_tuning_both_directions():
    h = mg.gen_rmat(12, 16, 44, symmetrize=False)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        for setting in BFS_SETTINGS[:4]:
            g.set_tuning(**{**mg.Graph.default_tuning(), **setting})
            for directed in (1, 0):
                d, _ = g.bfs([3], directed=directed)
                np.testing.assert_array_equal(d, oracle.bfs(h.row_offsets, h.col_idx, [3], directed=directed))


def test_autotune_caches_per_graph_class(tmp_path):
    from mirrorofmapgraph_b200 import tuning
    cache = str(tmp_path / "tuning.json")
    h = mg.gen_rmat(14, 16, 1001, symmetrize=True, weights="int", p0=1, p1=255)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        ent = tuning.tune(g, programs=("bfs", "sssp"), cache=cache, reps=1)
        assert not ent["cached"] and ent["class"] == tuning.graph_class(g)
        assert ent["class"].split("|")[1:] == ["n2^14", "deg2^5", ent["class"].split("|")[3], "sym", "w"]
        got = g.tuning()
        for prog in ("bfs", "sssp"):
            assert ent["times_ms"][prog][0] <= ent["times_ms"][prog][1]
            for f, vals in tuning.CANDIDATES[prog].items():
                assert got[f] in vals + [mg.Graph.default_tuning()[f]]
                assert ent["tuning"][f] == got[f]
        db = tuning.load_cache(cache)
        assert set(db[ent["class"]]["programs"]) == {"bfs", "sssp"}
        # the tuned graph is exact
        for s in (0, 5):
            np.testing.assert_array_equal(g.bfs([s])[0], oracle.bfs(h.row_offsets, h.col_idx, [s]))
            np.testing.assert_array_equal(g.sssp([s])[0], oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [s]))
    # another graph of the same class takes the cached setting without timing
    h2 = mg.gen_rmat(14, 16, 1002, symmetrize=True, weights="int", p0=1, p1=255)
    with mg.Graph(h2.row_offsets, h2.col_idx, h2.weights_i32, symmetric=True) as g2:
        if tuning.graph_class(g2) == ent["class"]:
            e2 = tuning.tune(g2, programs=("bfs",), cache=cache)
            assert e2["cached"] and all(g2.tuning()[f] == ent["tuning"][f] for f in ent["tuning"])
        g2.set_tuning(**mg.Graph.default_tuning())
        assert tuning.apply_cached(g2, cache) == (tuning.graph_class(g2) in db)
    # a batch program extends the class's entry
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True) as g:
        e3 = tuning.tune(g, programs=("sssp_batch",), sources=[0, 1, 2, 3, 4, 5, 6, 7], cache=cache, reps=1)
        assert not e3["cached"] and set(e3["programs"]) == {"bfs", "sssp", "sssp_batch"}
        assert g.tuning()["sssp_batch_heavy"] in tuning.CANDIDATES["sssp_batch"]["sssp_batch_heavy"]


def test_degree_stats(rmat13):
    import ctypes as C
    h, g = rmat13
    mx, iso = C.c_int64(), C.c_int64()
    assert g._lib.mg_graph_degree_stats(g._h, C.byref(mx), C.byref(iso)) == L.MG_OK
    deg = np.diff(h.row_offsets)
    assert mx.value == deg.max() and iso.value == int((deg == 0).sum())


@pytest.mark.parametrize("rounds", [0, 1, 2, 8])
def test_cc_rounds_are_exact(rounds):
    """Every count of neighbour-sampling rounds gives the minimum-id labels: a
    symmetric R-MAT graph (sampling over the CSR), a directed one read both ways
    (sampling over CSR and CSC) and a graph of many small components."""
    graphs = [(mg.gen_rmat(13, 16, 71, symmetrize=True), True), (mg.gen_rmat(12, 8, 72, symmetrize=False), False),
              (mg.gen_er(5000, 3000, 73), False)]
    for h, sym in graphs:
        with mg.Graph(h.row_offsets, h.col_idx, symmetric=sym) as g:
            g.set_tuning(cc_rounds=rounds)
            lab, st = g.cc()
            np.testing.assert_array_equal(lab, oracle.cc(h.row_offsets, h.col_idx))
            assert st["edges_traversed"] == h.m
