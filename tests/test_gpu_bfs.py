"""BFS on the GPU through the C ABI, bit-exact against the reference's CPUBFS
(golden vectors) and the oracle, in every direction mode and loop driver."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200 import _lib as L

pytestmark = pytest.mark.gpu

MODES = [dict(direction="push"), dict(direction="pull"), dict(direction="auto"),
         dict(direction="auto", use_graph=False)]


def _graph(d, symmetric=False, values=True):
    return mg.Graph(np.array(d["row_offsets"], dtype=np.int32), np.array(d["col_idx"], dtype=np.int32),
                    np.array(d["values"], dtype=np.int32) if values else None, symmetric=symmetric)


@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
@pytest.mark.parametrize("mode", MODES)
def test_bfs_fixtures(mtx_fixtures, name, mode):
    d = mtx_fixtures[name]
    with _graph(d) as g:
        depth, st = g.bfs([0], directed=1, **mode)
        assert depth.tolist() == d["cpubfs_directed"]
        if name == "chesapeake":
            depth, _ = g.bfs([0], directed=0, **mode)
            assert depth.tolist() == d["cpubfs_undirected"]


def test_bfs_chesapeake_readme_counts(mtx_fixtures):
    # README:55-75: the undirected chesapeake run visits 170 edges in 2 iterations.
    d = mtx_fixtures["chesapeake"]
    with _graph(d) as g:
        depth, st = g.bfs([0], directed=0, direction="push")
    assert max(depth) == 2


@pytest.mark.parametrize("mode", MODES)
def test_bfs_er_golden(synthetic_golden, mode):
    from golden.make_golden import er_graph
    G = synthetic_golden
    h = er_graph()
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        for i, s in enumerate(G["er_sources"]):
            depth, st = g.bfs([s], **mode)
            assert (depth == G["er_bfs"][i]).all()
            reached = depth >= 0
            assert st["edges_traversed"] == int(np.diff(h.row_offsets)[reached].sum())


@pytest.mark.parametrize("mode", MODES)
def test_bfs_rmat_golden(synthetic_golden, mode):
    from golden.make_golden import rmat_graph
    G = synthetic_golden
    h = rmat_graph()
    for sym in (False, True):
        with mg.Graph(h.row_offsets, h.col_idx, symmetric=sym) as g:
            for i, s in enumerate(G["rmat_sources"]):
                depth, _ = g.bfs([s], **mode)
                assert (depth == G["rmat_bfs"][i]).all()


@pytest.mark.parametrize("scale", [14, 17])
def test_bfs_rmat_vs_oracle(scale):
    h = mg.gen_rmat(scale, 16, 1234 + scale, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        for s in (0, 1, h.n // 2 + 3):
            ref = oracle.bfs(h.row_offsets, h.col_idx, [s])
            for mode in MODES:
                depth, st = g.bfs([s], **mode)
                assert (depth == ref).all(), mode
            depth, st = g.bfs([s], direction="auto")
            assert st["status_detail"] >= 0  # bottom-up levels run


def test_bfs_directed_rmat_pull_uses_csc():
    h = mg.gen_rmat(13, 8, 77, symmetrize=False)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        for s in (0, 5):
            ref = oracle.bfs(h.row_offsets, h.col_idx, [s])
            for mode in MODES:
                assert (g.bfs([s], **mode)[0] == ref).all()
            ref0 = oracle.bfs(h.row_offsets, h.col_idx, [s], directed=0)
            assert (g.bfs([s], directed=0)[0] == ref0).all()


def test_bfs_lattice():
    h = mg.gen_lattice(200, 150, 0.001, 9)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        ref = oracle.bfs(h.row_offsets, h.col_idx, [0])
        d1, st = g.bfs([0])
        d2, _ = g.bfs([0], use_graph=False)
        assert (d1 == ref).all() and (d2 == ref).all()
        assert st["iterations"] == ref.max() + 1


def test_bfs_multisource_and_duplicates():
    h = mg.gen_er(3000, 9000, 21)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        srcs = [5, 5, 17, 2999, 17]
        ref = oracle.bfs(h.row_offsets, h.col_idx, srcs)
        for mode in MODES:
            assert (g.bfs(srcs, **mode)[0] == ref).all()


def test_bfs_iter_num_caps_levels():
    h = mg.gen_er(2000, 5000, 3)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        full = oracle.bfs(h.row_offsets, h.col_idx, [0])
        for cap in (1, 2, 3):
            d, st = g.bfs([0], iter_num=cap)
            exp = np.where(full <= cap, full, -1)
            assert (d == exp).all() and st["iterations"] <= cap


def test_bfs_queue_overflow_reports_status():
    h = mg.gen_rmat(12, 16, 5, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        with pytest.raises(mg.MapGraphError) as e:
            g.bfs([0], queue_sizing=0.001, direction="push")
        assert e.value.status == L.MG_ERR_QUEUE_OVERFLOW
        # the graph stays usable after the error
        assert (g.bfs([0])[0] == oracle.bfs(h.row_offsets, h.col_idx, [0])).all()


def test_bfs_bad_arguments():
    h = mg.gen_er(100, 300, 3)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        for bad in ([-1], [100], [0, 1000]):
            with pytest.raises(mg.MapGraphError) as e:
                g.bfs(bad)
            assert e.value.status == L.MG_ERR_ARG


def test_graph_validation_rejects_bad_csr():
    with pytest.raises(mg.MapGraphError) as e:
        mg.Graph(np.array([0, 2, 1, 3], dtype=np.int32), np.array([0, 1, 2], dtype=np.int32))
    assert e.value.status == L.MG_ERR_ARG
    with pytest.raises(mg.MapGraphError) as e:
        mg.Graph(np.array([0, 1, 2], dtype=np.int32), np.array([0, 5], dtype=np.int32))
    assert e.value.status == L.MG_ERR_ARG


def test_edge_cases_tiny_graphs():
    # single vertex, no edges
    with mg.Graph(np.array([0, 0], dtype=np.int32), np.zeros(0, dtype=np.int32)) as g:
        assert g.bfs([0])[0].tolist() == [0]
    # isolated vertices and a self-loop
    ro = np.array([0, 1, 2, 2, 2], dtype=np.int32)
    ci = np.array([0, 0], dtype=np.int32)
    with mg.Graph(ro, ci) as g:
        assert g.bfs([1])[0].tolist() == [1, 0, -1, -1]
        assert g.bfs([1], directed=0)[0].tolist() == [1, 0, -1, -1]


def test_bfs_device_output_and_determinism():
    torch = pytest.importorskip("torch")
    h = mg.gen_rmat(15, 16, 8, symmetrize=True)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        out = torch.empty(h.n, dtype=torch.int32, device="cuda")
        _, st = g.bfs([0], out=out)
        ref = oracle.bfs(h.row_offsets, h.col_idx, [0])
        assert (out.cpu().numpy() == ref).all()
        a, _ = g.bfs([0])
        b, _ = g.bfs([0])
        assert (a == b).all()


def test_csc_build_matches_stable_transpose():
    torch = pytest.importorskip("torch")
    for scale, ef in ((11, 16), (14, 4), (12, 200)):
        h = mg.gen_rmat(scale, ef, 31, symmetrize=False)
        co, ri, perm = oracle.csc_of(h.row_offsets, h.col_idx)
        with mg.Graph(h.row_offsets, h.col_idx) as g:
            p = g.device_arrays()
            got = {}
            for key, count in (("col_offsets", h.n + 1), ("row_idx", h.m), ("csc_perm", h.m)):
                t = torch.empty(count, dtype=torch.int32, device="cuda")
                _copy_device_ptr(t, p[key])
                got[key] = t.cpu().numpy()
            assert (got["col_offsets"] == co).all()
            assert (got["row_idx"] == ri).all()
            assert (got["csc_perm"] == perm).all()


def _copy_device_ptr(dst_tensor, src_ptr):
    """Copies dst.numel() int32 values from a raw device pointer into a CUDA tensor."""
    import ctypes as C
    import torch
    nbytes = dst_tensor.numel() * 4
    cudart = C.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    rc = cudart.cudaMemcpy(C.c_void_p(dst_tensor.data_ptr()), C.c_void_p(src_ptr), nbytes, 3)
    assert rc == 0
    torch.cuda.synchronize()


@pytest.mark.parametrize("kind", ["rmat", "er"])
def test_bfs_predecessors_match_reference_rule(kind):
    torch = pytest.importorskip("torch")
    h = (mg.gen_rmat(12, 16, 31, symmetrize=False) if kind == "rmat" else mg.gen_er(5000, 20000, 3))
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        depth, _ = g.bfs([1])
        pred = g.bfs_predecessors(depth)
        ref = oracle.bfs_pred(h.row_offsets, h.col_idx, depth)
        np.testing.assert_array_equal(pred, ref)
        # every reached non-source vertex points one level up, along an edge
        rows = np.repeat(np.arange(h.n), np.diff(h.row_offsets))
        edges = set(zip(rows.tolist(), h.col_idx.tolist()))
        for v in np.flatnonzero(depth > 0)[:500]:
            u = pred[v]
            assert depth[u] == depth[v] - 1 and (int(u), int(v)) in edges
        dd = torch.from_numpy(depth).cuda()
        dp = torch.empty(h.n, dtype=torch.int32, device="cuda")
        g.bfs_predecessors(dd, out=dp)
        np.testing.assert_array_equal(dp.cpu().numpy(), ref)


@pytest.mark.parametrize("mode", MODES)
def test_bfs_long_lattice_persistent_levels(mode):
    # a 1024 x 512 lattice without shortcuts: about 1,500 levels of small
    # frontiers, run by the persistent cooperative kernel; directed=0 reads the
    # same edges from both sides
    h = mg.gen_lattice(1024, 512, 0.0, 4)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        depth, st = g.bfs([0], **mode)
        ref = oracle.bfs(h.row_offsets, h.col_idx, [0])
        np.testing.assert_array_equal(depth, ref)
        assert st["iterations"] == ref.max() + 1
        d2, _ = g.bfs([h.n - 1, 5], directed=0, **mode)
        np.testing.assert_array_equal(d2, oracle.bfs(h.row_offsets, h.col_idx, [h.n - 1, 5]))


def _csr_from_pairs(n, src, dst):
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    ro = np.zeros(n + 1, dtype=np.int32)
    np.add.at(ro, src + 1, 1)
    return np.cumsum(ro, dtype=np.int64).astype(np.int32), dst.astype(np.int32)


@pytest.mark.parametrize("mode", MODES)
def test_bfs_hubs_inside_small_push_levels(mode):
    # Hubs of 5,000-12,000 edges reached while the frontier is still small (the
    # persistent levels): a root with 6 hub children, each hub with its own
    # leaves, and a 300-vertex path hanging off one leaf. Hubs of >= 4096 edges
    # go to the grid-strided pass inside the persistent kernel.
    rng = np.random.default_rng(5)
    hubs = np.arange(1, 7)
    sizes = [5000, 12000, 4096, 4095, 7000, 9000]
    src, dst, nxt = [np.zeros(6, np.int64)], [hubs], 7
    for h_, k in zip(hubs, sizes):
        leaves = np.arange(nxt, nxt + k)
        nxt += k
        src.append(np.full(k, h_)); dst.append(rng.permutation(leaves))
    path = np.arange(nxt, nxt + 300)
    src.append(np.concatenate([[nxt - 1], path[:-1]])); dst.append(path)
    n = int(path[-1]) + 1
    s = np.concatenate(src); d = np.concatenate(dst)
    ro, ci = _csr_from_pairs(n, np.concatenate([s, d]), np.concatenate([d, s]))
    with mg.Graph(ro, ci, symmetric=True) as g:
        for srcs in ([0], [path[-1]], [3, path[150]]):
            ref = oracle.bfs(ro, ci, srcs)
            depth, st = g.bfs(srcs, **mode)
            np.testing.assert_array_equal(depth, ref)
            assert st["iterations"] == ref.max() + 1
            assert st["edges_traversed"] == int((ro[1:] - ro[:-1])[ref >= 0].sum())
