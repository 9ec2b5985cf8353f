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
