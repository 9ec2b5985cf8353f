"""Batched traversals on the GPU: mg_bfs_batch (bit-parallel, 64 sources per
group), mg_sssp_batch and mg_bfs_ragged, each row bit-exact against the oracle
and against the single-source engine entry points."""
import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg

pytestmark = pytest.mark.gpu


def _c4_sources(ro, k, seed):
    return mg.mixed_degree_sources(ro, k, seed)


@pytest.fixture(scope="module")
def rmat14():
    h = mg.gen_rmat(14, 16, 41, symmetrize=True, weights="int", p0=1, p1=255)
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True)
    yield h, g
    g.close()


@pytest.mark.parametrize("mode", [dict(direction="auto"), dict(direction="push"), dict(direction="pull"),
                                  dict(direction="auto", use_graph=False)])
def test_bfs_batch_64_matches_single_runs(rmat14, mode):
    h, g = rmat14
    srcs = _c4_sources(h.row_offsets, 64, 3)
    depth, st = g.bfs_batch(srcs, **mode)
    assert depth.shape == (64, h.n)
    etrav = 0
    for i, s in enumerate(srcs):
        one, s1 = g.bfs([int(s)], direction="push")
        np.testing.assert_array_equal(depth[i], one)
        etrav += s1["edges_traversed"]
    assert st["edges_traversed"] == etrav
    for i in (0, 33, 63):
        np.testing.assert_array_equal(depth[i], oracle.bfs(h.row_offsets, h.col_idx, [int(srcs[i])]))


def test_bfs_batch_groups_duplicates_and_unreached():
    # 70 sources = two groups; repeated sources; a directed graph with unreachable parts.
    h = mg.gen_er(3000, 6000, 17)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        rng = np.random.default_rng(5)
        srcs = rng.integers(0, h.n, 70).astype(np.int32)
        srcs[10] = srcs[11] = srcs[69]
        for directed in (1, 0):
            depth, _ = g.bfs_batch(srcs, directed=directed)
            csc = oracle.csc_of(h.row_offsets, h.col_idx)
            for i in range(70):
                ref = oracle.bfs(h.row_offsets, h.col_idx, [int(srcs[i])], directed=directed, csc=csc)
                np.testing.assert_array_equal(depth[i], ref)


def test_bfs_batch_device_output(rmat14):
    torch = pytest.importorskip("torch")
    h, g = rmat14
    srcs = np.arange(5, dtype=np.int32)
    out = torch.empty(5 * h.n, dtype=torch.int32, device="cuda")
    g.bfs_batch(srcs, out=out)
    host, _ = g.bfs_batch(srcs)
    np.testing.assert_array_equal(out.cpu().numpy().reshape(5, h.n), host)


def test_bfs_ragged_matches_each_member():
    rng = np.random.default_rng(9)
    members = [mg.gen_rmat(int(s), 8, 100 + i, symmetrize=True) for i, s in enumerate(rng.integers(6, 13, 12))]
    with mg.Graph.ragged(members, symmetric=True) as g:
        bases = g.ragged_bases()
        srcs = np.zeros(len(members), dtype=np.int32)
        depth, st = g.bfs_ragged(srcs)
        etrav = 0
        for i, hm in enumerate(members):
            ref = oracle.bfs(hm.row_offsets, hm.col_idx, [0])
            np.testing.assert_array_equal(depth[bases[i]:bases[i + 1]], ref)
            reached = ref >= 0
            etrav += int(np.diff(hm.row_offsets)[reached].sum())
        assert st["edges_traversed"] == etrav


def test_bfs_ragged_full_batch_32_graphs():
    """The batched workload's ragged batch at its stated size: 32 independent
    R-MAT graphs of scale U{10..18}, edge factor 8, symmetrised (the bench's own
    seeds), one BFS from vertex 0 each in one device run; every member bit-exact
    against the oracle's BFS of that graph alone (the reference runs one engine
    call per source, Algorithms/BFS/bfs.cu:442-456)."""
    seed = 20140601
    rng = np.random.default_rng(seed + 10)
    scales = rng.integers(10, 19, 32)
    members = [mg.gen_rmat(int(sc), 8, seed + 100 + i, symmetrize=True) for i, sc in enumerate(scales)]
    assert len(members) == 32 and scales.min() >= 10 and scales.max() <= 18
    with mg.Graph.ragged(members, symmetric=True) as g:
        bases = g.ragged_bases()
        for direction in ("auto", "push"):
            depth, st = g.bfs_ragged(np.zeros(32, dtype=np.int32), direction=direction)
            etrav = 0
            for i, hm in enumerate(members):
                ref = oracle.bfs(hm.row_offsets, hm.col_idx, [0])
                np.testing.assert_array_equal(depth[bases[i]:bases[i + 1]], ref)
                etrav += int(np.diff(hm.row_offsets)[ref >= 0].sum())
            assert st["edges_traversed"] == etrav


def test_bfs_ragged_rejects_bad_sources():
    members = [mg.gen_er(50, 200, 1), mg.gen_er(30, 90, 2)]
    with mg.Graph.ragged(members) as g:
        with pytest.raises(mg.MapGraphError):
            g.bfs_ragged(np.array([0, 30], dtype=np.int32))


@pytest.mark.parametrize("use_graph", [True, False])
def test_sssp_batch_64_matches_single_runs(rmat14, use_graph):
    h, g = rmat14
    srcs = _c4_sources(h.row_offsets, 64, 4)
    dist, st = g.sssp_batch(srcs, use_graph=use_graph)
    assert dist.shape == (64, h.n)
    etrav = 0
    for i, s in enumerate(srcs):
        one, s1 = g.sssp([int(s)])
        np.testing.assert_array_equal(dist[i], one)
        etrav += s1["edges_traversed"]
    assert st["edges_traversed"] == etrav
    for i in (0, 40):
        np.testing.assert_array_equal(dist[i], oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [int(srcs[i])]))


def test_sssp_batch_ragged_rows_and_outputs():
    # n = 3000 is not a power of two: rows are computed padded and packed.
    torch = pytest.importorskip("torch")
    h = mg.gen_er(3000, 9000, 23, weights="int", p0=1, p1=64)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        srcs = np.array([0, 7, 7, 2999, 1500], dtype=np.int32)
        csc = oracle.csc_of(h.row_offsets, h.col_idx)
        for directed in (1, 0):
            dist, _ = g.sssp_batch(srcs, directed=directed)
            dev = torch.empty(5 * h.n, dtype=torch.int32, device="cuda")
            g.sssp_batch(srcs, out=dev, directed=directed)
            np.testing.assert_array_equal(dev.cpu().numpy().reshape(5, h.n), dist)
            for i, s in enumerate(srcs):
                one, _ = g.sssp([int(s)], directed=directed)
                np.testing.assert_array_equal(dist[i], one)


def test_sssp_batch_power_of_two_device_output(rmat14):
    torch = pytest.importorskip("torch")
    h, g = rmat14
    srcs = np.array([1, 2, 3], dtype=np.int32)
    dev = torch.empty(3 * h.n, dtype=torch.int32, device="cuda")
    g.sssp_batch(srcs, out=dev)
    host, _ = g.sssp_batch(srcs)
    np.testing.assert_array_equal(dev.cpu().numpy().reshape(3, h.n), host)


@pytest.mark.parametrize("nsrc", [1, 31, 33, 70])
def test_sssp_batch_interleaved_rows(nsrc):
    """Mean out-degree above 8: the batch runs on interleaved distance rows (32
    instances per row, groups of 32). Every row equals the oracle's single-source
    distances, out- and in-edges, with repeated sources and zero weights."""
    torch = pytest.importorskip("torch")
    h = mg.gen_rmat(12, 16, 123, symmetrize=False, weights="int", p0=0, p1=40)
    assert h.m > 8 * h.n
    rng = np.random.default_rng(nsrc)
    srcs = rng.integers(0, h.n, nsrc).astype(np.int32)
    if nsrc > 3:
        srcs[1] = srcs[2]
    deg = np.diff(h.row_offsets).astype(np.int64)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_i32) as g:
        for directed in (1, 0):
            dist, st = g.sssp_batch(srcs, directed=directed)
            etrav = 0
            for i, s_ in enumerate(srcs):
                ref = oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [int(s_)], directed)
                np.testing.assert_array_equal(dist[i], ref)
                etrav += int(deg[ref < 2**31 - 1].sum())
            assert st["edges_traversed"] == etrav
            dev = torch.empty(nsrc * h.n, dtype=torch.int32, device="cuda")
            g.sssp_batch(srcs, out=dev, directed=directed, use_graph=False)
            np.testing.assert_array_equal(dev.cpu().numpy().reshape(nsrc, h.n), dist)
    with mg.Graph(h.row_offsets, h.col_idx) as g:  # unit weights: distance = BFS depth
        dist, _ = g.sssp_batch(srcs[:5])
        for i in range(min(5, nsrc)):
            bd = oracle.bfs(h.row_offsets, h.col_idx, [int(srcs[i])])
            np.testing.assert_array_equal(dist[i], np.where(bd < 0, 2**31 - 1, bd))


def _sparse_teleports(n, nvec, seed):
    return mg.sparse_teleports(n, nvec, seed)


PR_L1_TOL = 1e-6  # FP32 engine vs FP64 oracle, same iteration count


def _check_vectors(h, xs, tele, iters, which, weights=None):
    for k in which:
        xr, it, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, weights, 0.85, 0.0, iters,
                                         tele[k].astype(np.float64))
        assert it == iters
        err = np.abs(xs[k].astype(np.float64) - xr).sum()
        assert err <= PR_L1_TOL, (k, err)


def test_ppr_batch_256_vectors_with_hub_chunks():
    # scale 14 symmetric R-MAT has rows above the 2048-edge hub threshold
    h = mg.gen_rmat(14, 16, 77, symmetrize=True)
    assert np.diff(h.row_offsets).max() > 2048
    tele = _sparse_teleports(h.n, 256, 8)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        xs, st = g.pagerank(teleport=tele, nvec=256, mode="normalized")
        assert xs.shape == (256, h.n)
        assert st["residual"] < 1e-6 or st["iterations"] == 50
        assert st["edges_traversed"] == 256 * h.m * st["iterations"]
        np.testing.assert_allclose(xs.astype(np.float64).sum(axis=1), 1.0, atol=1e-5)
        _check_vectors(h, xs, tele, st["iterations"], [0, 1, 100, 200, 255])
        xs2, _ = g.pagerank(teleport=tele, nvec=256, mode="normalized", use_graph=False)
        assert np.abs(xs - xs2).sum() <= 1e-9 * 256


def test_ppr_batch_weighted_directed_and_device_output():
    torch = pytest.importorskip("torch")
    h = mg.gen_rmat(12, 16, 99, symmetrize=False, weights="lognormal", p0=0, p1=1)
    tele = _sparse_teleports(h.n, 40, 3)
    with mg.Graph(h.row_offsets, h.col_idx, h.weights_f32) as g:
        xs, st = g.pagerank(teleport=tele, nvec=40, mode="normalized", weighted=True)
        _check_vectors(h, xs, tele, st["iterations"], range(0, 40, 7), weights=h.weights_f32)
        td = torch.from_numpy(tele.reshape(-1)).cuda()
        out = torch.empty(40 * h.n, dtype=torch.float32, device="cuda")
        g.pagerank(teleport=td, nvec=40, out=out, mode="normalized", weighted=True)
        assert np.abs(out.cpu().numpy().reshape(40, h.n) - xs).sum() <= 1e-9 * 40


@pytest.mark.parametrize("nvec", [2, 33, 100, 300])
def test_ppr_batch_widths_and_groups(nvec):
    # fixed 25 iterations (tol 0) so every group of 256 runs the same schedule
    h = mg.gen_rmat(11, 8, 5, symmetrize=False)
    tele = _sparse_teleports(h.n, nvec, nvec)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        xs, st = g.pagerank(teleport=tele, nvec=nvec, mode="normalized", tol=1e-30, max_iter=25)
        assert st["iterations"] == 25
        _check_vectors(h, xs, tele, 25, sorted({0, nvec // 2, nvec - 1}))


@pytest.mark.parametrize("width", [32, 64, 128])
def test_ppr_group_width_and_autotuned_width(width):
    # Fixed 25 iterations: every group runs the same schedule whatever its width.
    h = mg.gen_rmat(12, 8, 7, symmetrize=True)
    tele = _sparse_teleports(h.n, 150, 11)
    with mg.Graph(h.row_offsets, h.col_idx, symmetric=True) as g:
        xs, st = g.pagerank(teleport=tele, nvec=150, mode="normalized", tol=1e-30, max_iter=25, group_width=width)
        assert st["status_detail"] == width and st["iterations"] == 25
        _check_vectors(h, xs, tele, 25, [0, width - 1, width, 149])
        xa, sa = g.pagerank(teleport=tele, nvec=150, mode="normalized", tol=1e-30, max_iter=25, autotune=True)
        assert sa["status_detail"] in (64, 128, 256)
        assert np.abs(xa - xs).sum() <= 1e-9 * 150
        with pytest.raises(mg.MapGraphError):
            g.pagerank(teleport=tele, nvec=150, mode="normalized", group_width=48)
