"""Batched workloads across ranks (one process per GPU, torch.distributed).

The instances of a batch -- BFS/SSSP sources, personalised PageRank vectors,
member graphs of a ragged batch -- are independent, so they shard without any
exchange during the run: every rank holds the whole graph, runs a contiguous
slice of the instances through the single-GPU batched entry point, and one
all-gather at the end assembles the full result on every rank. No reference
counterpart (the reference drives one GPU; its multi-GPU partitioning scaffolding,
GASengine/csr_problem.cuh:339-365, is unused).

With the NCCL backend the gather runs on device tensors; with gloo (CPU tests) on
host tensors. Slices are padded to the largest one so that every rank sends the
same number of rows, as all-gather needs.
"""
from __future__ import annotations

import numpy as np


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous slice [lo, hi) of `total` instances owned by `rank`: the first
    total % world ranks get one instance more."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    base, extra = divmod(int(total), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_rows(local: np.ndarray, total: int, group=None) -> np.ndarray:
    """All-gathers row slices (rank r holds rows shard_range(total, r, world))
    into the full `total x row` array on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = shard_range(total, rank, world)
    local = np.asarray(local)
    if local.shape[0] != hi - lo:
        raise ValueError(f"rank {rank} holds {local.shape[0]} rows, owns {hi - lo}")
    width = local.shape[1:]
    most = -(-int(total) // world)
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    pad = torch.zeros((most,) + tuple(width), dtype=torch.from_numpy(local[:0].copy()).dtype, device=dev)
    pad[: hi - lo] = torch.from_numpy(np.ascontiguousarray(local)).to(dev)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    rows = []
    for r in range(world):
        a, b = shard_range(total, r, world)
        rows.append(parts[r][: b - a].cpu().numpy())
    return np.concatenate(rows, axis=0)


def bfs_batch_sharded(graph, srcs, group=None, **kw) -> np.ndarray:
    """Depth rows (len(srcs) x n) of a multi-source BFS with the sources split
    over the ranks; every rank returns the full array."""
    import torch.distributed as dist

    srcs = np.asarray(srcs, dtype=np.int32)
    lo, hi = shard_range(srcs.size, dist.get_rank(group), dist.get_world_size(group))
    local = graph.bfs_batch(srcs[lo:hi], **kw)[0] if hi > lo else np.zeros((0, graph.n), np.int32)
    return gather_rows(local, srcs.size, group)


def sssp_batch_sharded(graph, srcs, group=None, **kw) -> np.ndarray:
    """Distance rows (len(srcs) x n) with the sources split over the ranks."""
    import torch.distributed as dist

    srcs = np.asarray(srcs, dtype=np.int32)
    lo, hi = shard_range(srcs.size, dist.get_rank(group), dist.get_world_size(group))
    local = graph.sssp_batch(srcs[lo:hi], **kw)[0] if hi > lo else np.zeros((0, graph.n), np.int32)
    return gather_rows(local, srcs.size, group)


def pagerank_sharded(graph, teleport: np.ndarray, group=None, **kw) -> np.ndarray:
    """Personalised PageRank rows (nvec x n) with the teleport vectors split over
    the ranks (each rank runs its slice as one batched solve)."""
    import torch.distributed as dist

    teleport = np.asarray(teleport, dtype=np.float32)
    nvec = teleport.shape[0]
    lo, hi = shard_range(nvec, dist.get_rank(group), dist.get_world_size(group))
    kw.setdefault("mode", "normalized")
    if hi - lo == 0:
        local = np.zeros((0, graph.n), np.float32)
    else:
        x, _ = graph.pagerank(teleport=np.ascontiguousarray(teleport[lo:hi]), nvec=hi - lo, **kw)
        local = np.asarray(x).reshape(hi - lo, graph.n)
    return gather_rows(local, nvec, group)


def ragged_partition(sizes, world: int) -> list[list[int]]:
    """Member indices per rank for a ragged batch: longest first, each to the
    least-loaded rank (ties to the lower rank), so the largest per-rank load is
    within one member of the best split; each rank's list is in member order.
    Deterministic, so every rank computes the same partition without talking."""
    if world <= 0:
        raise ValueError(f"world of {world}")
    sizes = [int(s) for s in sizes]
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def _all_gather_1d(local: np.ndarray, lengths: list[int], group=None) -> list[np.ndarray]:
    """All-gathers one 1-D int32 array per rank (rank r's has lengths[r] entries,
    known to every rank) padded to the longest; returns the unpadded arrays."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    most = max(1, max(lengths))
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    pad = torch.zeros(most, dtype=torch.int32, device=dev)
    if local.size:
        pad[: local.size] = torch.from_numpy(np.ascontiguousarray(local, dtype=np.int32)).to(dev)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return [parts[r][: lengths[r]].cpu().numpy() for r in range(world)]


def bfs_ragged_sharded(members, srcs, group=None, symmetric: bool = False, make_graph=None, **kw):
    """BFS of every member graph of a ragged batch from its source srcs[i], the
    members split over the ranks (ragged_partition by vertices + edges): each rank
    uploads only its members as one ragged graph (Graph.ragged, or
    make_graph(members, symmetric=...)) and runs one mg_bfs_ragged; one
    all-gather assembles every member's depth array on every rank. Returns
    (depths, stats): depths[i] is member i's depth array, stats holds the summed
    edges_traversed, the largest per-rank kernel_ms, and members_per_rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    srcs = np.asarray(srcs, dtype=np.int32)
    if srcs.size != len(members):
        raise ValueError(f"{srcs.size} sources for {len(members)} member graphs")
    nv = [int(np.asarray(m.row_offsets).size) - 1 for m in members]
    parts = ragged_partition([nv[i] + int(np.asarray(members[i].col_idx).size) for i in range(len(members))], world)
    mine = parts[rank]
    edges, ms = 0.0, 0.0
    local = np.zeros(0, np.int32)
    if mine:
        if make_graph is None:
            from .graph import Graph
            make_graph = Graph.ragged
        g = make_graph([members[i] for i in mine], symmetric=symmetric)
        try:
            depth, st = g.bfs_ragged(srcs[mine], **kw)
        finally:
            g.close()
        local = np.asarray(depth, dtype=np.int32)
        edges, ms = float(st["edges_traversed"]), float(st["kernel_ms"])
    lengths = [sum(nv[i] for i in parts[r]) for r in range(world)]
    if local.size != lengths[rank]:
        raise ValueError(f"rank {rank}: ragged BFS returned {local.size} depths for {lengths[rank]} vertices")
    chunks = _all_gather_1d(local, lengths, group)
    depths: list = [None] * len(members)
    for r in range(world):
        off = 0
        for i in parts[r]:
            depths[i] = chunks[r][off:off + nv[i]]
            off += nv[i]
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    t = torch.tensor([edges], dtype=torch.float64, device=dev)
    dist.all_reduce(t, group=group)
    tm = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX, group=group)
    return depths, {"edges_traversed": float(t.item()), "kernel_ms": float(tm.item()),
                    "members_per_rank": [len(p) for p in parts]}
