"""BFS and PageRank over a 1-D vertex partition on the GPU (mg_part_* through the
C ABI): slices of one graph run as separate partitions on one GPU, exchanging
through a shared buffer, and as a one-rank NCCL group. BFS depths bit-exact
against the oracle and the single-GPU BFS, levels and traversed edges equal;
PageRank within 1e-6 L1 of the FP64 oracle at the same iteration count, and the
same iteration count as the single-GPU solver."""
import os
import socket

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200.partition import (CollectiveExchange, GraphSlice, bfs_partitioned,
                                             bfs_partitioned_local, pagerank_partitioned,
                                             pagerank_partitioned_local, partition_cuts)

PR_L1_TOL = 1e-6  # FP32 slices vs the FP64 oracle at the same iteration count

pytestmark = pytest.mark.gpu


def _slices(h, world, symmetric=False):
    c = partition_cuts(h.row_offsets, world)
    return [GraphSlice.from_csr(h.row_offsets, h.col_idx, int(c[r]), int(c[r + 1]), symmetric=symmetric)
            for r in range(world)]


def _check(h, srcs, world, mode, symmetric=False):
    ref = oracle.bfs(h.row_offsets, h.col_idx, srcs)
    parts = _slices(h, world, symmetric)
    try:
        d, st = bfs_partitioned_local(parts, srcs, direction=mode)
        np.testing.assert_array_equal(d, ref)
        assert st["iterations"] == ref.max() + 1
        assert st["edges_traversed"] == int(np.diff(h.row_offsets)[ref >= 0].sum())
        for p in parts[1:]:
            np.testing.assert_array_equal(p.result()[0], ref)
        return st
    finally:
        for p in parts:
            p.close()


@pytest.mark.parametrize("world", [1, 2, 3, 4])
@pytest.mark.parametrize("mode", ["auto", "push", "pull"])
def test_partitioned_bfs_rmat_directed(world, mode):
    h = mg.gen_rmat(14, 8, 9)
    st = _check(h, [0, 123, 4095], world, mode)
    if mode == "pull":
        assert st["status_detail"] == st["iterations"] - 1


@pytest.mark.parametrize("world", [2, 5])
def test_partitioned_bfs_symmetric_and_hubs(world):
    h = mg.gen_rmat(15, 16, 4, symmetrize=True)
    deg = np.diff(h.row_offsets)
    hub = int(np.argmax(deg))
    assert deg[hub] >= 4096  # the grid-strided pass of the push step
    _check(h, [hub], world, "push", symmetric=True)
    _check(h, [hub, 77], world, "auto", symmetric=True)


def test_partitioned_bfs_lattice_many_levels():
    h = mg.gen_lattice(120, 90, 0.0, 3)
    st = _check(h, [0], 3, "auto", symmetric=True)
    assert st["iterations"] > 200


def test_partitioned_matches_single_gpu_and_iter_cap():
    h = mg.gen_er(5000, 30000, 8)
    with mg.Graph(h.row_offsets, h.col_idx) as g:
        d1, s1 = g.bfs([3])
    parts = _slices(h, 3)
    try:
        d2, s2 = bfs_partitioned_local(parts, [3])
        np.testing.assert_array_equal(d1, d2)
        assert s1["iterations"] == s2["iterations"] and s1["edges_traversed"] == s2["edges_traversed"]
        d3, s3 = bfs_partitioned_local(parts, [3], iter_num=2)
        np.testing.assert_array_equal(d3, np.where((d1 >= 0) & (d1 <= 2), d1, -1))
        assert s3["iterations"] == 2
    finally:
        for p in parts:
            p.close()


def test_slice_rejects_bad_layouts():
    h = mg.gen_er(100, 300, 2)
    with pytest.raises(mg.MapGraphError):
        GraphSlice.from_csr(h.row_offsets, h.col_idx, 10, 64)  # lo not a multiple of 32
    bad = h.col_idx.copy()
    bad[5] = 100
    with pytest.raises(mg.MapGraphError):
        GraphSlice.from_csr(h.row_offsets, bad, 0, 100)  # vertex id out of range
    with GraphSlice.from_csr(h.row_offsets, h.col_idx, 0, 100) as p:
        with pytest.raises(mg.MapGraphError):
            p.begin([100])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partitioned_bfs_over_a_one_rank_nccl_group():
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        h = mg.gen_rmat(13, 8, 12)
        ref = oracle.bfs(h.row_offsets, h.col_idx, [1])
        with GraphSlice.from_csr(h.row_offsets, h.col_idx, 0, h.n) as p:
            d, st = bfs_partitioned(p, [1], CollectiveExchange())
            np.testing.assert_array_equal(d, ref)
            out = torch.empty(h.n, dtype=torch.int32, device="cuda")
            d2, _ = bfs_partitioned(p, [1], CollectiveExchange(), out=out)
            np.testing.assert_array_equal(out.cpu().numpy(), ref)
            x, st = pagerank_partitioned(p, [0, h.n], CollectiveExchange())
            xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
            assert np.abs(x - xr).sum() <= PR_L1_TOL
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [1, 2, 3, 4])
@pytest.mark.parametrize("symmetric", [True, False])
def test_partitioned_pagerank_matches_oracle_and_single_gpu(world, symmetric):
    h = mg.gen_rmat(14, 8, 21, symmetrize=symmetric)
    c = partition_cuts(h.row_offsets, world)
    parts = _slices(h, world, symmetric)
    try:
        x, st = pagerank_partitioned_local(parts, c)
        xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
        assert np.abs(x - xr).sum() <= PR_L1_TOL
        for p in parts[1:]:
            np.testing.assert_array_equal(p.pr_result()[0], x)
        with mg.Graph(h.row_offsets, h.col_idx, symmetric=symmetric) as g:
            xs, ss = g.pagerank(mode="normalized", alpha=0.85, tol=1e-6, max_iter=50)
        assert ss["iterations"] == st["iterations"]
        assert np.abs(x - xs).sum() <= PR_L1_TOL
        assert st["residual"] < 1e-6 or st["iterations"] == 50
        x3, s3 = pagerank_partitioned_local(parts, c, max_iter=3)
        assert s3["iterations"] == 3
        xr3, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, 3)
        assert np.abs(x3 - xr3).sum() <= PR_L1_TOL
    finally:
        for p in parts:
            p.close()


def test_partitioned_pagerank_hub_rows_and_protocol_errors():
    h = mg.gen_rmat(15, 16, 4, symmetrize=True)  # rows of >= 2,048 edges: chunked hub rows
    assert np.diff(h.row_offsets).max() >= 4096
    c = partition_cuts(h.row_offsets, 3)
    parts = _slices(h, 3, True)
    try:
        x, st = pagerank_partitioned_local(parts, c)
        xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, None, 0.85, 0.0, st["iterations"])
        assert np.abs(x - xr).sum() <= PR_L1_TOL
        import torch
        buf = torch.zeros(h.n, dtype=torch.float32, device="cuda")
        with pytest.raises(mg.MapGraphError):
            parts[0].pr_merge(buf, 1, h.n, [0, h.n])  # no step pending
        parts[0].pr_begin()
        parts[0].pr_step(buf)
        with pytest.raises(mg.MapGraphError):
            parts[0].pr_step(buf)  # step twice
        with pytest.raises(mg.MapGraphError):
            parts[0].pr_merge(buf, 1, h.n, [0, h.n])  # cuts without this slice's range
    finally:
        for p in parts:
            p.close()
