"""BFS over a 1-D vertex partition on the GPU (mg_part_* through the C ABI):
slices of one graph run as separate partitions on one GPU, exchanging through a
shared buffer, and as a one-rank NCCL group; depths bit-exact against the
oracle and the single-GPU BFS, levels and traversed edges equal."""
import os
import socket

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200.partition import (CollectiveExchange, GraphSlice, bfs_partitioned,
                                             bfs_partitioned_local, partition_cuts)

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
    finally:
        dist.destroy_process_group()
