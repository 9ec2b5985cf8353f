"""Sharding of batched workloads over ranks (host logic, CPU): two gloo ranks
split sources / teleport vectors, run their slice, and all-gather the rows. The
per-rank compute is a deterministic stand-in with the Graph method signatures,
so the test needs no GPU."""
import os
import socket

import numpy as np
import pytest

from mirrorofmapgraph_b200.sharding import shard_range


def test_shard_range_covers_every_instance_once():
    for total in (0, 1, 5, 64, 100):
        for world in (1, 2, 3, 8):
            spans = [shard_range(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and b >= a
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


class _FakeGraph:
    """Deterministic stand-in for mirrorofmapgraph_b200.Graph (same signatures)."""
    n = 11

    def bfs_batch(self, srcs, **kw):
        srcs = np.asarray(srcs, np.int32)
        return (np.add.outer(srcs, np.arange(self.n)) % 7).astype(np.int32), {}

    def sssp_batch(self, srcs, **kw):
        srcs = np.asarray(srcs, np.int32)
        return (np.add.outer(3 * srcs, np.arange(self.n)) % 1000).astype(np.int32), {}

    def pagerank(self, teleport=None, nvec=1, **kw):
        t = np.asarray(teleport, np.float32).reshape(nvec, self.n)
        return (2 * t + 0.5).reshape(-1) if nvec == 1 else 2 * t + 0.5, {}


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from mirrorofmapgraph_b200 import sharding
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = _FakeGraph()
        srcs = np.arange(9, dtype=np.int32) * 5
        tele = np.random.default_rng(0).random((7, g.n)).astype(np.float32)
        d = sharding.bfs_batch_sharded(g, srcs)
        s = sharding.sssp_batch_sharded(g, srcs)
        p = sharding.pagerank_sharded(g, tele)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), d=d, s=s, p=p)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batches_gather_full_results(tmp_path, world):
    import torch.multiprocessing as mp
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    g = _FakeGraph()
    srcs = np.arange(9, dtype=np.int32) * 5
    tele = np.random.default_rng(0).random((7, g.n)).astype(np.float32)
    for r in range(world):
        z = np.load(tmp_path / f"r{r}.npz")
        np.testing.assert_array_equal(z["d"], g.bfs_batch(srcs)[0])
        np.testing.assert_array_equal(z["s"], g.sssp_batch(srcs)[0])
        np.testing.assert_array_equal(z["p"], g.pagerank(tele, nvec=7)[0])


def test_ragged_partition_balances_and_covers():
    from mirrorofmapgraph_b200.sharding import ragged_partition
    rng = np.random.default_rng(3)
    for k in (1, 5, 32):
        sizes = rng.integers(1, 1 << 12, k)
        for world in (1, 2, 3, 8):
            parts = ragged_partition(sizes, world)
            assert sorted(i for p in parts for i in p) == list(range(k))
            assert all(p == sorted(p) for p in parts)
            loads = [int(sizes[p].sum()) if p else 0 for p in parts]
            assert max(loads) - min(loads) <= int(sizes.max())  # LPT: within one member
            assert parts == ragged_partition(sizes, world)  # deterministic


class _FakeRagged:
    """Stand-in for Graph.ragged: the union of the members, BFS by the oracle."""

    def __init__(self, members, symmetric=False):
        self.members = members

    def bfs_ragged(self, srcs, **kw):
        import oracle
        parts, edges = [], 0
        for m, s in zip(self.members, srcs):
            d = oracle.bfs(m.row_offsets, m.col_idx, [int(s)])
            parts.append(d)
            edges += int(np.diff(m.row_offsets)[d >= 0].sum())
        return np.concatenate(parts).astype(np.int32), {"edges_traversed": edges, "kernel_ms": float(len(parts))}

    def close(self):
        pass


def _ragged_members():
    import mirrorofmapgraph_b200 as mg
    rng = np.random.default_rng(11)
    return [mg.gen_rmat(int(sc), 8, 500 + i, symmetrize=True) for i, sc in enumerate(rng.integers(4, 10, 7))]


def _ragged_worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from mirrorofmapgraph_b200 import sharding
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        members = _ragged_members()
        srcs = np.array([i % 3 for i in range(len(members))], dtype=np.int32)
        depths, st = sharding.bfs_ragged_sharded(members, srcs, symmetric=True, make_graph=_FakeRagged)
        np.savez(os.path.join(out_dir, f"g{rank}.npz"), *depths, edges=st["edges_traversed"], ms=st["kernel_ms"],
                 per=np.array(st["members_per_rank"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 8])
def test_ragged_bfs_sharded_gathers_every_member(tmp_path, world):
    import torch.multiprocessing as mp
    import oracle
    mp.start_processes(_ragged_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    members = _ragged_members()
    refs = [oracle.bfs(m.row_offsets, m.col_idx, [i % 3]) for i, m in enumerate(members)]
    edges = sum(int(np.diff(m.row_offsets)[r >= 0].sum()) for m, r in zip(members, refs))
    for r in range(world):
        z = np.load(tmp_path / f"g{r}.npz")
        for i, ref in enumerate(refs):
            np.testing.assert_array_equal(z[f"arr_{i}"], ref)
        assert float(z["edges"]) == edges
        per = z["per"].tolist()
        assert sum(per) == len(members) and len(per) == world
        assert float(z["ms"]) == max(per)  # the stand-in's time is its member count: max over ranks
