"""Autotuner for the traversal thresholds and launch shapes (mg_tuning).

The reference fixes its expansion and contraction tile shapes at compile time
(GASengine/vertex_centric/*_problem_type.cuh, one CTA/warp/thread split for
every graph). Here each field of ``mg_tuning`` is read by the kernels at every
call, so the best setting can follow the graph: :func:`tune` times candidate
values on the device (the engine's own CUDA-event ``kernel_ms``), one field at a
time from the current setting (coordinate descent; a value is kept only when it
beats the incumbent by ``min_gain``), applies the winner to the graph and caches
it in a JSON file under the graph's class. :func:`apply_cached` reuses a cached
setting for another graph of the same class without timing anything.

A graph's class is the GPU name, log2 of its vertex count, log2 of its mean
out-degree, log2 of the ratio of its largest to its mean out-degree (the skew:
R-MAT hubs against lattices and uniform graphs), whether it is symmetric and
whether it carries edge weights.
"""
from __future__ import annotations

import json
import math
import os
import time
from typing import Callable, Iterable, Sequence

import numpy as np

# Candidate values per field, grouped by the program whose time decides them.
CANDIDATES: dict[str, dict[str, list[int]]] = {
    "bfs": {
        "bfs_cta_th": [256, 512, 1024, 2048],
        "bfs_grid_th": [2048, 4096, 8192, 16384],
        "bfs_defer_warp": [0, 1],
        "bfs_persist_max": [0, 1 << 14, 1 << 16, 1 << 18],
        "bfs_persist_edges": [1 << 15, 1 << 17, 1 << 19],
        "bfs_alpha": [8, 14, 24],
        "bfs_beta": [12, 24, 48],
        "bfs_ctas_per_sm": [2, 4, 8],
        "bfs_tail_max": [0, 512, 2048, 8192],
        "bfs_tail_edges": [4096, 16384, 65536],
    },
    "sssp": {
        "sssp_heavy": [64, 128, 256, 512],
        "sssp_heavy_small": [16, 32, 64],
        "sssp_ctas_per_sm": [2, 4],
    },
    "sssp_batch": {
        "sssp_batch_heavy": [16, 32, 64, 128],
    },
    "cc": {
        "cc_rounds": [0, 1, 2, 3],
    },
}

# Fields whose legal range depends on another field: set the bound first.
_ORDER_AFTER = {"sssp_heavy_small": "sssp_heavy"}


def default_cache_path() -> str:
    """$MG_TUNING_CACHE, else ~/.cache/mirrorofmapgraph_b200/tuning.json."""
    env = os.environ.get("MG_TUNING_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "mirrorofmapgraph_b200", "tuning.json")


def _gpu_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(torch.cuda.current_device())
    except Exception:
        pass
    return "gpu"


def class_key(n: int, m: int, max_degree: int, symmetric: bool, weighted: bool, gpu: str | None = None) -> str:
    """The cache key of a graph class (see the module docstring)."""
    mean = m / max(1, n)
    lg = lambda x: int(round(math.log2(x))) if x > 0 else 0  # noqa: E731
    skew = lg(max_degree / mean) if mean > 0 else 0
    return (f"{gpu if gpu is not None else _gpu_name()}|n2^{lg(n)}|deg2^{lg(mean)}|skew2^{skew}|"
            f"{'sym' if symmetric else 'dir'}|{'w' if weighted else 'u'}")


def graph_class(graph) -> str:
    """class_key of a device graph (its out-degree statistics come from the device)."""
    from . import _lib as L
    import ctypes as C
    mx, iso = C.c_int64(), C.c_int64()
    st = graph._lib.mg_graph_degree_stats(graph._h, C.byref(mx), C.byref(iso))
    if st != L.MG_OK:
        from .graph import _check
        _check(st, "mg_graph_degree_stats")
    weighted = bool(graph.device_arrays()["edge_vals"])
    return class_key(graph.n, graph.m, mx.value, bool(graph.flags & L.MG_GRAPH_SYMMETRIC), weighted)


def load_cache(path: str | None = None) -> dict:
    p = path or default_cache_path()
    try:
        with open(p) as f:
            db = json.load(f)
        return db if isinstance(db, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(db: dict, path: str | None = None) -> None:
    p = path or default_cache_path()
    d = os.path.dirname(p)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = p + f".tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def _default_sources(graph, k: int, seed: int = 7, tries: int = 64) -> list[int]:
    """k sources whose BFS reaches a large part of the graph (a timing from an
    isolated vertex says nothing about the thresholds): up to `tries` seeded random
    vertices are run once each, and the k that traverse the most edges are kept,
    in the order they were drawn (deterministic for a graph)."""
    rng = np.random.default_rng(seed)
    cand = [int(s) for s in rng.integers(0, max(1, graph.n), tries)]
    reach = []
    for s in cand:
        reach.append(graph.bfs([s])[1]["edges_traversed"])
        if sum(r >= graph.m // 4 for r in reach) >= k:  # enough sources in the large component
            break
    best = sorted(range(len(reach)), key=lambda i: (-reach[i], i))[:k]
    return [cand[i] for i in sorted(best)]


def device_time(graph, program: str, sources: Sequence[int], reps: int = 3) -> float:
    """Median over reps of the summed device time (ms) of one run per source of
    `program` ("bfs", "sssp" single-source, "sssp_batch" one batch of all
    sources, "cc" one run per source, which it does not use), after one untimed
    run (plans, loop graphs)."""
    import torch
    out = torch.empty(graph.n * (len(sources) if program == "sssp_batch" else 1), dtype=torch.int32,
                      device="cuda")

    def once() -> float:
        if program == "sssp_batch":
            return graph.sssp_batch(np.asarray(sources, dtype=np.int32), out=out)[1]["kernel_ms"]
        if program == "cc":
            return sum(graph.cc(out=out)[1]["kernel_ms"] for _ in sources)
        fn = graph.bfs if program == "bfs" else graph.sssp
        return sum(fn([s], out=out)[1]["kernel_ms"] for s in sources)

    once()
    return float(np.median([once() for _ in range(reps)]))


def search(start: dict, programs: Iterable[str], measure: Callable[[str, dict], float], min_gain: float = 0.02,
           valid: Callable[[dict], bool] | None = None) -> tuple[dict, dict]:
    """Coordinate descent from `start`: for each program and each of its fields,
    time every candidate value with the other fields fixed and keep the fastest
    when it beats the incumbent by more than `min_gain` (a fraction). `measure(
    program, setting)` returns a time; `valid(setting)` screens settings out of
    range. Returns (setting, {program: [best time, default time]})."""
    cur = dict(start)
    times: dict[str, list[float]] = {}
    for prog in programs:
        fields = CANDIDATES[prog]
        base = measure(prog, cur)
        first = base
        for field in sorted(fields, key=lambda f: (f in _ORDER_AFTER, f)):
            best_v, best_t = cur[field], base
            for v in fields[field]:
                if v == cur[field]:
                    continue
                trial = {**cur, field: v}
                if valid is not None and not valid(trial):
                    continue
                t = measure(prog, trial)
                if t < best_t * (1.0 - min_gain):
                    best_v, best_t = v, t
            cur[field] = best_v
            base = best_t
        times[prog] = [base, first]
    return cur, times


def tune(graph, programs: Sequence[str] = ("bfs", "sssp"), sources: Sequence[int] | None = None,
         cache: str | None = None, force: bool = False, reps: int = 3, min_gain: float = 0.02) -> dict:
    """Tunes `graph` for `programs` (keys of CANDIDATES) and applies the result.
    With a cached entry for the graph's class (and force=False) the cached setting
    is applied without timing. Returns the cache entry: {"tuning", "programs",
    "times_ms" ({program: [tuned, default]}), "class", "cached" (True when it came
    from the cache)}."""
    key = graph_class(graph)
    db = load_cache(cache)
    ent = db.get(key)
    if ent and not force and set(programs) <= set(ent.get("programs", [])):
        graph.set_tuning(**{**graph.tuning(), **ent["tuning"]})
        return {**ent, "class": key, "cached": True}
    if sources is None:
        sources = _default_sources(graph, 4)
    from .graph import MapGraphError

    def valid(setting: dict) -> bool:
        saved = graph.tuning()
        try:
            graph.set_tuning(**setting)
            return True
        except MapGraphError:
            return False
        finally:
            graph.set_tuning(**saved)

    def measure(prog: str, setting: dict) -> float:
        graph.set_tuning(**setting)
        return device_time(graph, prog, sources, reps)

    start = graph.tuning()
    t0 = time.time()
    best, times = search(start, programs, measure, min_gain, valid)
    graph.set_tuning(**best)
    # the tuned programs' fields, over what the class already had for others
    tuned = {f: best[f] for prog in programs for f in CANDIDATES[prog]}
    old = (ent or {}) if not force else {}
    ent = {"tuning": {**old.get("tuning", {}), **tuned},
           "programs": sorted(set(programs) | set(old.get("programs", []))),
           "times_ms": {**old.get("times_ms", {}), **times}, "search_s": time.time() - t0,
           "sources": [int(s) for s in sources]}
    db[key] = ent
    save_cache(db, cache)
    return {**ent, "class": key, "cached": False}


def apply_cached(graph, cache: str | None = None) -> bool:
    """Applies the cached setting of the graph's class, if any; returns whether
    one was found."""
    ent = load_cache(cache).get(graph_class(graph))
    if not ent:
        return False
    graph.set_tuning(**{**graph.tuning(), **ent["tuning"]})
    return True
