#!/usr/bin/env python3
"""Benchmark of the GAS engine on one B200 per rank.

Workload (R-MAT scale 22, edge factor 16, a/b/c/d = 0.57/0.19/0.19/0.05, no vertex
permutation, symmetrised, int32 CSR, weights U{1..255}, seeded synthetic graph):
one step runs, on the device-resident graph,

  BFS from a seeded source  -> TEPS edges = sum of out-degrees of reached vertices
  CC                        -> TEPS edges = m
  PageRank (normalised, alpha 0.85, L1 residual < 1e-6 or 50 iterations)
                            -> TEPS edges = m * iterations

value = sum of TEPS edges / sum of their device times (GTEPS, CUDA events on the
engine's stream, L2 flushed between steps). SSSP is timed after the steps, reported
under "per_algorithm", and folded into "value_all_four" (all four programs per
step); the headline leaves it out because the reference's CPU SSSP is O(n^2) and
has no CPU baseline at this size.

--impl reference times the reference's own CPU functions (CPUBFS, CPUCC, CPUPR,
compiled from the reference tree into oracle/_ref) on the host, on the same
scale-22 graph, the driver's passes divided among the host cores.

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torch.distributed.run (one replica per GPU, no data-path collective: every rank
runs the full workload on its own graph, "scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS (BFS + CC + PageRank aggregate, R-MAT s22 ef16 symmetric)"
SEED = 20140601
ALPHA, PR_TOL, PR_MAX_IT = 0.85, 1e-6, 50
CPU_SAMPLE_SCALE = 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--e2e-steps", type=int, default=10)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample-scale", type=int, default=CPU_SAMPLE_SCALE,
                   help="R-MAT scale of the bounded sample of the GPU arm's one-core cpu_baseline")
    p.add_argument("--ref-scale", type=int, default=None,
                   help="R-MAT scale the reference arm runs on (default: --scale, the headline graph)")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-versus-looped section")
    p.add_argument("--no-tune", action="store_true",
                   help="keep the default traversal tuning (otherwise the BFS/SSSP/CC thresholds are tuned on "
                        "the device for the graph's class before the warm-up, or taken from the JSON cache)")
    p.add_argument("--batched-scale", type=int, default=20)
    p.add_argument("--pr-gather", default="auto", choices=["auto", "binned", "cached", "tma", "segmented"],
                   help="PageRank gather: autotuned per graph (default) or forced (for profiling one kernel)")
    p.add_argument("--no-extra", action="store_true",
                   help="skip the lattice (BFS/SSSP) and weighted PageRank forward + adjoint sections")
    p.add_argument("--host-loop", action="store_true",
                   help="drive iterations from the host instead of a CUDA-graph WHILE node (for profilers "
                        "that cannot see kernels inside conditional graphs)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# Kernels of one PageRank iteration per gather variant (mg_stats.variant).
PR_KERNELS = {0: "solve_binned_kernel", 1: "solve_gather_kernel + solve_fixup_kernel",
              2: "solve_binned_hub_kernel", 3: "solve_segment_kernel + solve_rows_kernel"}


def pagerank_fp64_check(h, x_gpu, iters, weights=None, fixed_point=True):
    """Error of a GPU PageRank result against the FP64 oracle: L1 at the same
    number of iterations (the tests' 1e-6 bound), and, when asked, L1 to the FP64
    fixed point (power iteration to an L1 change below 1e-11). Part of the CPU
    baseline leg: the oracle is the checker, outside every timed region."""
    import oracle
    t0 = time.perf_counter()
    xr, _, _ = oracle.pr_normalized(h.row_offsets, h.col_idx, weights, ALPHA, 0.0, int(iters))
    out = {"l1_vs_fp64": float(np.abs(x_gpu.astype(np.float64) - xr).sum()), "iterations": int(iters),
           "tolerance": PR_TOL}
    if fixed_point:
        xf, itf, rf = oracle.pr_normalized(h.row_offsets, h.col_idx, weights, ALPHA, 1e-11, 1000)
        out["l1_vs_fp64_fixed_point"] = float(np.abs(x_gpu.astype(np.float64) - xf).sum())
        out["fixed_point_iterations"] = int(itf)
    out["check_s"] = time.perf_counter() - t0
    return out


def sources(h, k, seed):
    deg = np.diff(h.row_offsets)
    cand = np.flatnonzero(deg > 0)
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.choice(cand, size=k, replace=False)]


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        # raw samples: $MG_CLOCK_LOG (a directory) if set, else a temporary file
        log_dir = os.environ.get("MG_CLOCK_LOG")
        self.path = os.path.join(log_dir, f"clocks_rank{device_index}.csv") if log_dir and os.path.isdir(log_dir) \
            else f"/tmp/mg_clocks_{os.getpid()}_{device_index}.csv"

    def _lines(self) -> int:
        try:
            with open(self.path) as f:
                return sum(1 for ln in f if ln.endswith("\n"))
        except OSError:
            return 0

    def start(self):
        """Starts sampling every 50 ms and waits (up to 5 s) for the first sample,
        so that the sampler is running when the timed region begins."""
        self.mark_at = 0
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while self._lines() == 0 and time.time() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.02)

    def mark(self):
        """The timed region starts: samples from here on are the region's."""
        self.mark_at = self._lines()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        # a region shorter than the sampling period still gets the first sample after it began
        t0 = time.time()
        while self._lines() <= self.mark_at and time.time() - t0 < 1.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for i, line in enumerate(open(self.path)):
            if i < self.mark_at:
                continue
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def batched_section(scale, torch, mg, tune=True):
    """Batched workload against looping the plain engine once per instance, on
    the same GPU: 64 BFS and 64 SSSP sources (half top-1% degree, half median
    degree), 256 personalised PageRank vectors (supports of U{1..32} vertices)
    on R-MAT `scale` ef16 symmetrised with weights U{1..255}, and a ragged batch
    of 32 R-MAT graphs of scale U{10..18} (ef 8), one BFS from vertex 0 each.
    Device time from the engine's CUDA events; TEPS edges per instance as in the
    plain runs (PPR: m x iterations per vector)."""
    h = mg.gen_rmat(scale, 16, SEED + 7, symmetrize=True, weights="int", p0=1, p1=255)
    n = h.n
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True)
    srcs = mg.mixed_degree_sources(h.row_offsets, 64, SEED + 8)
    out = torch.empty(64 * n, dtype=torch.int32, device="cuda")
    one = torch.empty(n, dtype=torch.int32, device="cuda")
    res = {}
    if tune:
        # both arms on the tuned setting: single-source BFS/SSSP (looped) and the batch
        from mirrorofmapgraph_b200 import tuning
        tuning.tune(g, programs=("bfs", "sssp"), sources=[int(s_) for s_ in srcs[:8]], reps=2)
        ent = tuning.tune(g, programs=("sssp_batch",), sources=[int(s_) for s_ in srcs], reps=2)
        res["tuning"] = {"class": ent["class"], "cached": ent["cached"], "tuning": ent["tuning"]}

    def pair(name, batched, looped, reps=2):
        # both arms warmed up once (plans, executable graphs), then timed
        for _ in range(reps):
            eb, tb = batched()
        looped()
        el, tl = looped()
        res[name] = {"batched_gteps": eb / tb / 1e6, "looped_gteps": el / tl / 1e6, "batched_ms": tb,
                     "looped_ms": tl, "speedup_gteps": (eb / tb) / (el / tl), "speedup_time": tl / tb}
        return eb, tb, el, tl

    def bfs_b():
        _, st = g.bfs_batch(srcs, out=out)
        return st["edges_traversed"], st["kernel_ms"]

    def bfs_l():
        e = t = 0.0
        for s_ in srcs:
            _, st = g.bfs([int(s_)], out=one)
            e += st["edges_traversed"]
            t += st["kernel_ms"]
        return e, t

    def sssp_b():
        _, st = g.sssp_batch(srcs, out=out)
        return st["edges_traversed"], st["kernel_ms"]

    def sssp_l():
        e = t = 0.0
        for s_ in srcs:
            _, st = g.sssp([int(s_)], out=one)
            e += st["edges_traversed"]
            t += st["kernel_ms"]
        return e, t

    tele = torch.from_numpy(mg.sparse_teleports(n, 256, SEED + 9).reshape(-1)).cuda()
    pout = torch.empty(256 * n, dtype=torch.float32, device="cuda")
    pone = torch.empty(n, dtype=torch.float32, device="cuda")

    # Both arms autotuned: the batch's group width, the single solves' gather.
    tuned = {}

    def ppr_b():
        _, st = g.pagerank(teleport=tele, nvec=256, out=pout, mode="normalized", alpha=ALPHA, tol=PR_TOL,
                           max_iter=PR_MAX_IT, autotune=True)
        tuned["group_width"] = st["status_detail"]
        return st["edges_traversed"], st["kernel_ms"]

    def ppr_l():
        e = t = 0.0
        for k in range(256):
            _, st = g.pagerank(teleport=tele[k * n:(k + 1) * n], out=pone, mode="normalized", alpha=ALPHA,
                               tol=PR_TOL, max_iter=PR_MAX_IT, autotune=True)
            e += st["edges_traversed"]
            t += st["kernel_ms"]
        return e, t

    tot = [0.0, 0.0, 0.0, 0.0]
    for name, b, l_ in (("bfs_64", bfs_b, bfs_l), ("sssp_64", sssp_b, sssp_l), ("ppr_256", ppr_b, ppr_l)):
        r = pair(name, b, l_)
        tot = [x + y for x, y in zip(tot, r)]
    res["ppr_256"]["group_width"] = tuned.get("group_width")
    g.close()
    rng = np.random.default_rng(SEED + 10)
    members = [mg.gen_rmat(int(sc), 8, SEED + 100 + i, symmetrize=True) for i, sc in enumerate(rng.integers(10, 19, 32))]
    gr = mg.Graph.ragged(members, symmetric=True)
    singles = [mg.Graph(m_.row_offsets, m_.col_idx, symmetric=True) for m_ in members]

    def rag_b():
        _, st = gr.bfs_ragged(np.zeros(32, dtype=np.int32))
        return st["edges_traversed"], st["kernel_ms"]

    def rag_l():
        e = t = 0.0
        for gm in singles:
            _, st = gm.bfs([0])
            e += st["edges_traversed"]
            t += st["kernel_ms"]
        return e, t

    r = pair("ragged_bfs_32", rag_b, rag_l)
    tot = [x + y for x, y in zip(tot, r)]
    gr.close()
    for gm in singles:
        gm.close()
    res["aggregate"] = {"batched_gteps": tot[0] / tot[1] / 1e6, "looped_gteps": tot[2] / tot[3] / 1e6,
                        "speedup_gteps": (tot[0] / tot[1]) / (tot[2] / tot[3])}
    res["config"] = (f"R-MAT s{scale} ef16 sym (n={n}, m={h.m}), weights U{{1..255}}; 64 BFS + 64 SSSP sources "
                     "(32 top-1% degree, 32 median); 256 PPR vectors (support U{1..32}); 32 ragged R-MAT graphs "
                     "scale U{10..18} ef8, BFS from 0; looped = one plain engine call per instance")
    return res


def sharded_section(scale, torch, mg, tune=True):
    """The batched workload split over the ranks (mirrorofmapgraph_b200.sharding,
    one process per GPU, no exchange during the runs): the ragged batch of 32 R-MAT
    graphs of scale U{10..18} (ef 8, BFS from vertex 0; members balanced over the
    ranks by size, each rank uploads only its own), and 64 BFS and 64 SSSP sources
    on R-MAT `scale` (every rank holds the graph and runs its slice of the sources
    as one batch). Device time = the largest per-rank kernel time (max over ranks);
    the all-gather that assembles every result on every rank is timed apart by
    the wall clock (max over ranks). Every rank returns the same dict."""
    import torch.distributed as dist
    from mirrorofmapgraph_b200 import sharding
    world = dist.get_world_size()
    dev = torch.device("cuda", torch.cuda.current_device())

    def max_over_ranks(x):
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    res = {"ranks": world}
    rng = np.random.default_rng(SEED + 10)
    members = [mg.gen_rmat(int(sc), 8, SEED + 100 + i, symmetrize=True) for i, sc in enumerate(rng.integers(10, 19, 32))]
    zeros = np.zeros(len(members), dtype=np.int32)
    for _ in range(2):  # the second run is timed (the first builds plans and loop graphs)
        dist.barrier()
        t0 = time.perf_counter()
        depths, st = sharding.bfs_ragged_sharded(members, zeros, symmetric=True)
        wall = max_over_ranks((time.perf_counter() - t0) * 1e3)
    res["ragged_bfs_32"] = {"gteps": st["edges_traversed"] / st["kernel_ms"] / 1e6, "kernel_ms": st["kernel_ms"],
                            "wall_ms_with_gather": wall, "members_per_rank": st["members_per_rank"],
                            "reached": int(sum(int((d >= 0).sum()) for d in depths))}
    h = mg.gen_rmat(scale, 16, SEED + 7, symmetrize=True, weights="int", p0=1, p1=255)
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True)
    if tune:
        from mirrorofmapgraph_b200 import tuning
        tuning.tune(g, programs=("bfs", "sssp", "sssp_batch"), sources=[0, 1, 2, 3], reps=2)
    srcs = mg.mixed_degree_sources(h.row_offsets, 64, SEED + 8)
    for name, fn in (("bfs_64", g.bfs_batch), ("sssp_64", g.sssp_batch)):
        lo, hi = sharding.shard_range(64, dist.get_rank(), world)
        for _ in range(2):
            dist.barrier()
            st = fn(srcs[lo:hi])[1] if hi > lo else {"kernel_ms": 0.0, "edges_traversed": 0}
            ms = max_over_ranks(st["kernel_ms"])
            e = torch.tensor([float(st["edges_traversed"])], dtype=torch.float64, device=dev)
            dist.all_reduce(e)
            t0 = time.perf_counter()
            rows = (sharding.bfs_batch_sharded if name == "bfs_64" else sharding.sssp_batch_sharded)(g, srcs)
            wall = max_over_ranks((time.perf_counter() - t0) * 1e3)
        res[name] = {"gteps": float(e.item()) / ms / 1e6 if ms else None, "kernel_ms": ms,
                     "wall_ms_sharded_call": wall, "rows": int(rows.shape[0])}
    g.close()
    res["config"] = (f"32 ragged R-MAT graphs scale U{{10..18}} ef8 (BFS from 0), and 64 BFS + 64 SSSP sources on "
                     f"R-MAT s{scale} ef16 sym weights U{{1..255}}, split over {world} ranks; kernel_ms = max over "
                     "ranks of the device time; the sharded call's wall time includes the all-gather")
    return res


def lattice_section(torch, mg, side=4096):
    """High-diameter workload: side x side 4-neighbour lattice (id = r * side + c)
    plus 0.1% uniform long-range pairs, every edge both ways, weights U{1..1000};
    BFS and SSSP from the corner vertex 0 (device time, CUDA events)."""
    h = mg.gen_lattice(side, side, 0.001, SEED + 11, weights="int", p0=1, p1=1000)
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True)
    out = torch.empty(h.n, dtype=torch.int32, device="cuda")
    res = {"config": f"lattice {side}x{side} + 0.1% long-range (n={h.n}, m={h.m}), weights U{{1..1000}}, src 0"}
    for name, fn in (("bfs", g.bfs), ("sssp", g.sssp)):
        for _ in range(2):
            _, st = fn([0], out=out)
        res[name] = {"gteps": st["edges_traversed"] / st["kernel_ms"] / 1e6, "ms": st["kernel_ms"],
                     "iterations": st["iterations"], "launches": st["launches"]}
    g.close()
    return res


def adjoint_section(torch, mg, scale=24, keep=None):
    """Weighted PageRank forward + adjoint: R-MAT `scale` ef16 directed, weights
    lognormal(0, 1) (normalised by their row sums), alpha 0.85, forward to L1 <
    1e-6 (gather autotuned per graph); backward of L = w . x with w ~ N(0, 1) to
    relative tolerance 1e-7. `keep` (a dict) receives the graph and the forward
    result for the FP64 check of the CPU baseline leg."""
    h = mg.gen_rmat(scale, 16, SEED + 12, symmetrize=False, weights="lognormal", p0=0, p1=1)
    n, m = h.n, h.m
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_f32)
    x = torch.empty(n, dtype=torch.float32, device="cuda")
    wv = torch.from_numpy(np.random.default_rng(SEED + 13).standard_normal(n).astype(np.float32)).cuda()
    gw = torch.empty(m, dtype=torch.float32, device="cuda")
    gt = torch.empty(n, dtype=torch.float32, device="cuda")
    for _ in range(2):
        _, sf = g.pagerank(mode="normalized", weighted=True, alpha=ALPHA, tol=PR_TOL, max_iter=200, out=x,
                           autotune=True)
        _, _, sb = g.pagerank_backward(x, wv, weighted=True, alpha=ALPHA, tol=1e-7, max_iter=200,
                                       out_weights=gw, out_teleport=gt)
    g.close()
    if keep is not None:
        keep.update(h=h, x=x.cpu().numpy(), iterations=sf["iterations"])
    return {"config": f"R-MAT s{scale} ef16 directed (n={n}, m={m}), lognormal(0,1) weights, alpha {ALPHA}",
            "forward": {"ms": sf["kernel_ms"], "iterations": sf["iterations"],
                        "gteps": m * sf["iterations"] / sf["kernel_ms"] / 1e6,
                        "gather_kernel": PR_KERNELS.get(sf["variant"])},
            "backward": {"ms": sb["kernel_ms"], "iterations": sb["iterations"],
                         "gteps": m * sb["iterations"] / sb["kernel_ms"] / 1e6}}


def cpu_reference_run(h, src):
    """One pass of the reference's CPU functions (BFS from src, CC, PageRank)."""
    import oracle
    R = oracle.Ref
    csc = (h.row_offsets, h.col_idx, None)  # symmetric: CSC = CSR
    deg = np.diff(h.row_offsets).astype(np.int64)
    d, tb = R.bfs(h.row_offsets, h.col_idx, src, 1, csc)
    eb = int(deg[d >= 0].sum())
    _, tc = R.cc(h.row_offsets, h.col_idx, csc)
    _, tp, sweeps = R.pr(h.row_offsets, h.col_idx, csc, with_sweeps=True)
    return {"bfs": (eb, tb), "cc": (h.m, tc), "pagerank": (h.m * max(sweeps, 0), tp), "pr_sweeps": sweeps}


def host_info() -> dict:
    """Host cores and CPU model (the CPU figures are quoted with them)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        ncores = len(os.sched_getaffinity(0))
    except Exception:
        ncores = os.cpu_count() or 1
    return {"nproc": ncores, "cpu_model": model}


def cpu_restatements(hs, src) -> dict:
    """Timed FP64/int restatements (oracle/) of the paths the reference has no CPU
    code for at these sizes, on the CPU sample graph, single-threaded: Dijkstra
    SSSP (the reference's CPUSSSP is O(n^2): hours at scale 22), one personalised
    PageRank vector and the PageRank adjoint."""
    import oracle
    out = {}
    t0 = time.perf_counter()
    d = oracle.sssp(hs.row_offsets, hs.col_idx, hs.weights_i32, [src])
    t = time.perf_counter() - t0
    deg = np.diff(hs.row_offsets).astype(np.int64)
    out["sssp_dijkstra"] = {"gteps": float(deg[d < 2**31 - 1].sum()) / t / 1e9, "s": t,
                            "kind": "restatement (heap Dijkstra, int32)"}
    tele = np.zeros(hs.n)
    tele[np.random.default_rng(SEED + 3).choice(hs.n, 16, replace=False)] = 1.0 / 16
    t0 = time.perf_counter()
    x, it, _ = oracle.pr_normalized(hs.row_offsets, hs.col_idx, None, ALPHA, PR_TOL, PR_MAX_IT, teleport=tele)
    t = time.perf_counter() - t0
    out["ppr_vector"] = {"gteps": hs.m * it / t / 1e9, "s": t, "iterations": int(it),
                         "kind": "restatement (FP64 power iteration)"}
    wv = np.random.default_rng(SEED + 4).standard_normal(hs.n)
    t0 = time.perf_counter()
    _, _, _, ita = oracle.pr_adjoint(hs.row_offsets, hs.col_idx, None, x, wv, ALPHA, 1e-9, 400)
    t = time.perf_counter() - t0
    out["pagerank_adjoint"] = {"gteps": hs.m * ita / t / 1e9, "s": t, "iterations": int(ita),
                               "kind": "restatement (FP64 adjoint solve + edge gradients)"}
    return out


def cpu_sample_graph(scale=CPU_SAMPLE_SCALE):
    import mirrorofmapgraph_b200 as mg
    return mg.gen_rmat(scale, 16, SEED, symmetrize=True, weights="int", p0=1, p1=255)


def reference_cpu_baseline(scale: int) -> dict:
    """`cpu_baseline` of the GPU arm: the reference's serial CPUBFS + CPUCC + CPUPR
    (oracle/_ref) once on the R-MAT sample of the given scale, one core, plus the
    FP64 / Dijkstra restatements timed beside them."""
    try:
        import oracle
        if not oracle.have_ref():
            return {"value": None, "unavailable": "oracle/_ref not built"}
        hs = cpu_sample_graph(scale)
        src = sources(hs, 1, SEED + 1)[0]
        r = cpu_reference_run(hs, src)
        ce = sum(r[k][0] for k in ("bfs", "cc", "pagerank"))
        cs = sum(r[k][1] for k in ("bfs", "cc", "pagerank"))
        return {
            "value": ce / cs / 1e9, "unit": "GTEPS", "cores": 1, "kind": "reference",
            "sample": f"reference CPUBFS + CPUCC + CPUPR (serial, oracle/_ref) once on R-MAT scale "
                      f"{scale} (same generator); {cs:.1f} s of CPU work",
            "per_algorithm": {k: r[k][0] / r[k][1] / 1e9 for k in ("bfs", "cc", "pagerank")},
            "host": host_info(),
            "sssp": "reference CPUSSSP not run: O(n^2), hours at scale 22 (timed at the 4,096-vertex "
                    "ER case in the tests); see restatements",
            "restatements": cpu_restatements(hs, src)}
    except Exception as e:
        return {"value": None, "unavailable": f"{type(e).__name__}: {e}"}


def _ref_worker(path, warm_srcs, timed_srcs, barrier, out):
    """One reference process: loads the graph, runs its share of the warm-up
    passes, waits for the others, then times its share of the timed passes of
    CPUBFS + CPUCC + CPUPR (one BFS source per pass)."""
    import mirrorofmapgraph_b200 as mg
    h = mg.load_csr(path)
    for s_ in warm_srcs:
        cpu_reference_run(h, s_)
    barrier.wait()
    t0 = time.time()
    per = {"bfs": [0, 0.0], "cc": [0, 0.0], "pagerank": [0, 0.0]}
    for s_ in timed_srcs:
        r = cpu_reference_run(h, s_)
        for k in per:
            per[k][0] += r[k][0]
            per[k][1] += r[k][1]
    out.put((t0, time.time(), per, len(timed_srcs)))


def run_reference(args):
    """The reference's own CPU implementation of the path (CPUBFS, CPUCC, CPUPR,
    compiled from the reference tree into oracle/_ref), on the GPU arm's graph
    (R-MAT --scale, same generator and seed). The functions are serial, so the
    host cores run independent processes; the driver's --warmup and --steps passes
    are divided among them (pass j goes to process j mod P and uses the GPU arm's
    BFS source of step j). The value is the timed passes' TEPS edges over the wall
    time from the common start to the last finish."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    t_all = time.time()
    try:
        import multiprocessing as mp
        import tempfile
        import oracle
        import mirrorofmapgraph_b200 as mg
        if not oracle.have_ref():
            raise RuntimeError("oracle/_ref/libmgref.so missing (reference CPU path not built)")
        sc = args.ref_scale if args.ref_scale else args.scale
        h = cpu_sample_graph(sc)
        try:
            ncores = len(os.sched_getaffinity(0))
        except Exception:
            ncores = os.cpu_count() or 1
        steps = max(1, args.steps)
        procs = max(1, min(32, ncores, steps))
        srcs = sources(h, max(steps + args.warmup, 8), SEED + 1)
        warm = [[srcs[j] for j in range(args.warmup) if j % procs == i] for i in range(procs)]
        timed = [[srcs[args.warmup + j] for j in range(steps) if j % procs == i] for i in range(procs)]
        tmpdir = tempfile.mkdtemp(prefix="mg_ref_")
        path = os.path.join(tmpdir, "graph.csr")
        mg.save_csr(path, h)
        ctx = mp.get_context("spawn")
        barrier, out = ctx.Barrier(procs), ctx.Queue()
        ps = [ctx.Process(target=_ref_worker, args=(path, warm[i], timed[i], barrier, out)) for i in range(procs)]
        for p_ in ps:
            p_.start()
        res = [out.get() for _ in ps]
        for p_ in ps:
            p_.join()
        os.remove(path)
        os.rmdir(tmpdir)
        busy = [r for r in res if r[3] > 0]
        wall = max(r[1] for r in busy) - min(r[0] for r in busy)
        per = {k: [sum(r[2][k][0] for r in res), sum(r[2][k][1] for r in res)] for k in ("bfs", "cc", "pagerank")}
        edges = sum(v[0] for v in per.values())
        value = edges / wall / 1e9
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32",
            "data": "synthetic (seeded R-MAT)",
            "config": {"workload": f"rmat_s{sc}_ef{args.edge_factor}_sym: CPUBFS + CPUCC + CPUPR",
                       "scale": sc, "edge_factor": 16, "n": h.n, "m": h.m},
            "host": host_info(),
            "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": procs, "kind": "reference",
                             "sample": f"the driver's {steps} timed step(s) (one BFS source each, CC, PageRank) "
                                       f"on R-MAT scale {sc}, divided among {procs} processes of the "
                                       f"reference's serial CPUBFS/CPUCC/CPUPR (pass j on process j mod "
                                       f"{procs}); {args.warmup} warm-up pass(es) divided the same way"},
            "per_algorithm": {k: {"gteps_per_core": v[0] / v[1] / 1e9 if v[1] else None, "core_seconds": v[1]}
                              for k, v in per.items()},
            "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": time.time() - t_all,
        }
    except Exception as e:  # the reference path could not run here
        line = {"impl": "reference", "unavailable": f"{type(e).__name__}: {e}"}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import mirrorofmapgraph_b200 as mg

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    peak, peak_kind = peaks()

    h = mg.gen_rmat(args.scale, args.edge_factor, SEED, symmetrize=True, weights="int", p0=1, p1=255)
    n, m = h.n, h.m
    srcs = sources(h, max(args.steps + args.warmup, 8), SEED + 1)
    g = mg.Graph(h.row_offsets, h.col_idx, h.weights_i32, symmetric=True)
    tune_info = None
    if not args.no_tune:
        # mirrorofmapgraph_b200.tuning: device-timed choice of the BFS/SSSP/CC thresholds
        # for this graph's class (or the cached one), before anything is timed
        from mirrorofmapgraph_b200 import tuning
        ent = tuning.tune(g, programs=("bfs", "sssp", "cc"), sources=[int(s_) for s_ in srcs[:4]], reps=3)
        tune_info = {"class": ent["class"], "cached": ent["cached"], "tuning": ent["tuning"],
                     "times_ms_tuned_vs_default": ent["times_ms"]}
    stream = torch.cuda.ExternalStream(g.stream_ptr)
    depth = torch.empty(n, dtype=torch.int32, device="cuda")
    label = torch.empty(n, dtype=torch.int32, device="cuda")
    rank_v = torch.empty(n, dtype=torch.float32, device="cuda")
    dist_v = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    deg = np.diff(h.row_offsets).astype(np.int64)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    ug = not args.host_loop

    pr_kw = dict(autotune=True) if args.pr_gather == "auto" else dict(gather=args.pr_gather)

    def step(i):
        with torch.cuda.stream(stream):
            flush.zero_()
        s = srcs[i % len(srcs)]
        (_, st_b), tb = timed(lambda: g.bfs([s], out=depth, use_graph=ug))
        (_, st_c), tc = timed(lambda: g.cc(out=label))
        # autotune: the first (warm-up) solve times the gather variants on this GPU
        # and graph and keeps the fastest (mg_pr_opts.autotune)
        (_, st_p), tp = timed(lambda: g.pagerank(mode="normalized", alpha=ALPHA, tol=PR_TOL, max_iter=PR_MAX_IT,
                                                 out=rank_v, use_graph=ug, **pr_kw))
        return {"bfs": (st_b["edges_traversed"], tb, st_b), "cc": (m, tc, st_c),
                "pagerank": (m * st_p["iterations"], tp, st_p)}

    clocks = Clocks(local)
    clocks.start()  # running before the timed region starts (its first sample can take a while)
    for i in range(args.warmup):
        step(i)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.mark()
    per = {"bfs": [0, 0.0], "cc": [0, 0.0], "pagerank": [0, 0.0]}
    launches = 0
    pr_iters = 0
    pr_cache = 0
    pr_variant = 0
    pr_last_iters = 0
    pr_ms = 0.0
    bfs_stats = []
    cc_stats = []
    for i in range(args.steps):
        r = step(args.warmup + i)
        for k in per:
            per[k][0] += r[k][0]
            per[k][1] += r[k][1]
            launches += r[k][2]["launches"]
        pr_iters += r["pagerank"][2]["iterations"]
        pr_cache = r["pagerank"][2]["status_detail"]
        pr_variant = r["pagerank"][2]["variant"]
        pr_last_iters = r["pagerank"][2]["iterations"]
        pr_ms += r["pagerank"][1]
        bfs_stats.append(r["bfs"][2])
        cc_stats.append(r["cc"][2])
    torch.cuda.synchronize()
    clock_info = clocks.stop()
    x_pr = rank_v.cpu().numpy()  # the last step's PageRank, for the FP64 check
    if dist:
        dist.barrier()
    edges = sum(v[0] for v in per.values())
    ms = sum(v[1] for v in per.values())
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        e = torch.tensor([float(edges)], dtype=torch.float64, device="cuda")
        dist.all_reduce(e)
        edges = float(e.item())
    value = edges / (ms * 1e-3) / 1e9

    # SSSP, reported per algorithm (not in the headline; see the module docstring).
    # One untimed run first (plans, the loop's executable graph).
    g.sssp([srcs[0]], out=dist_v, use_graph=ug)
    sssp_edges = sssp_ms = sssp_bytes = 0.0
    for i in range(min(3, args.steps)):
        with torch.cuda.stream(stream):
            flush.zero_()
        (_, st), t = timed(lambda: g.sssp([srcs[i]], out=dist_v, use_graph=ug))
        sssp_edges += st["edges_traversed"]
        sssp_ms += t
        sssp_bytes += st["bytes_compulsory"]

    # Roofline of the dominant kernel: one PageRank iteration of the gather the
    # autotuner kept (mg_stats.variant): solve_binned_kernel, solve_binned_hub_kernel
    # (column cache), or the segmented gather's pair solve_segment_kernel (hub rows
    # by column block) + solve_rows_kernel (the other rows, hub finishing, row
    # updates). Algorithmic bytes per iteration = offsets 4(n+1) + indices 4m +
    # read x 4n + write x 4n + write x/s 4n. Its duration is the PageRank call's
    # device time divided by the iterations (the call also holds a few init
    # kernels, so this slightly understates the kernels' own rate).
    pr_kernel = PR_KERNELS.get(pr_variant, "solve_binned_kernel")
    pr_bytes_iter = 4 * (n + 1) + 4 * m + 12 * n
    pr_s_iter = (pr_ms / max(pr_iters, 1)) * 1e-3
    achieved = pr_bytes_iter / pr_s_iter / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        t = tj.get(pr_kernel, {})
        if t.get("scale") == args.scale:
            traffic = t.get("dram_bytes_per_launch")
    except Exception:
        pass
    per_alg = {k: {"gteps": v[0] / (v[1] * 1e-3) / 1e9, "ms_per_run": v[1] / args.steps} for k, v in per.items()}
    per_alg["sssp"] = {"gteps": sssp_edges / (sssp_ms * 1e-3) / 1e9 if sssp_ms else None,
                       "ms_per_run": sssp_ms / max(1, min(3, args.steps)), "in_headline": False}
    # compulsory-byte roofline fractions per algorithm: the programs' own count of
    # compulsory DRAM bytes (mg_stats.bytes_compulsory) over their device time
    for k, sts in (("bfs", bfs_stats), ("cc", cc_stats)):
        bc = sum(s_["bytes_compulsory"] for s_ in sts)
        per_alg[k]["hbm_frac"] = bc / (per[k][1] * 1e-3) / 1e9 / peak
    if sssp_ms:
        per_alg["sssp"]["hbm_frac"] = sssp_bytes / (sssp_ms * 1e-3) / 1e9 / peak
    per_alg["pagerank"]["hbm_frac"] = achieved / peak
    per_alg["pagerank"]["gather_kernel"] = pr_kernel
    # All four programs per step: the three of the headline plus one SSSP run
    # (the mean of the SSSP runs above), on the same graph.
    nss = max(1, min(3, args.steps))
    value_all_four = None
    if sssp_ms:
        value_all_four = ((edges / args.steps + sssp_edges / nss) /
                          ((ms / args.steps + sssp_ms / nss) * 1e-3) / 1e9 * (world if world > 1 else 1))

    # End to end through the public API with host buffers: upload from pinned host
    # memory, run the three programs with outputs in pinned host buffers (read back
    # by each call), release the graph. One untimed pass first.
    ro_pin = torch.from_numpy(h.row_offsets).pin_memory()
    ci_pin = torch.from_numpy(h.col_idx).pin_memory()
    depth_pin = torch.empty(n, dtype=torch.int32).pin_memory()
    label_pin = torch.empty(n, dtype=torch.int32).pin_memory()
    rank_pin = torch.empty(n, dtype=torch.float32).pin_memory()
    e2e_edges = 0.0
    e2e_s = 0.0
    h2d = (n + 1) * 4 + m * 4
    d2h = 3 * n * 4
    # Pipelined like a stream of graphs: each step enqueues the next graph's
    # upload (asynchronous create) and then runs the three programs on the graph
    # uploaded by the previous step, so the PCIe copy overlaps the kernels; every
    # timed step still holds one full upload and the three read-backs.
    e2e_serial_s = 0.0
    if args.e2e_steps > 0:
        tuned = g.tuning() if tune_info else None

        def new_graph(**kw):
            gr = mg.Graph(ro_pin, ci_pin, symmetric=True, **kw)
            if tuned:
                gr.set_tuning(**tuned)
            return gr

        ge = new_graph(async_upload=True)
        for i in range(-1, args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            nxt = new_graph(async_upload=True)
            _, sb = ge.bfs([srcs[i % len(srcs)]], out=depth_pin)
            _, sc = ge.cc(out=label_pin)
            _, sp = ge.pagerank(mode="normalized", alpha=ALPHA, tol=PR_TOL, max_iter=PR_MAX_IT, out=rank_pin)
            ge.close()
            ge = nxt
            if i < 0:
                continue
            e2e_s += time.perf_counter() - t0
            e2e_edges += sb["edges_traversed"] + m + m * sp["iterations"]
        ge.close()
        # the same steps one graph at a time (upload, programs, release), for reference
        for i in range(-1, args.e2e_steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            with new_graph() as gs:
                gs.bfs([srcs[i % len(srcs)]], out=depth_pin)
                gs.cc(out=label_pin)
                gs.pagerank(mode="normalized", alpha=ALPHA, tol=PR_TOL, max_iter=PR_MAX_IT, out=rank_pin)
            if i >= 0:
                e2e_serial_s += time.perf_counter() - t0
    e2e = e2e_edges / e2e_s / 1e9 * (world if world > 1 else 1) if e2e_s > 0 else None

    line = {
        "metric": METRIC, "value": value, "value_all_four": value_all_four, "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32 (BFS/CC), f32 + f64 reductions (PageRank)",
        "data": "synthetic (seeded R-MAT, no vertex permutation)",
        "config": {"workload": f"rmat_s{args.scale}_ef{args.edge_factor}_sym: BFS + CC + PageRank(normalized, "
                               f"alpha {ALPHA}, tol {PR_TOL}, <= {PR_MAX_IT} it)",
                   "scale": args.scale, "edge_factor": args.edge_factor, "n": n, "m": m,
                   "l2": "256 MiB buffer written between steps; graph (CSR 537 MB) larger than L2",
                   "parallelism": f"replica x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "kernel": f"{pr_kernel} (one PageRank iteration per launch pair)"
                     if pr_variant in (1, 3) else f"{pr_kernel} (one PageRank iteration"
                     + (f", {pr_cache} cached columns)" if pr_cache else ")"),
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": pr_bytes_iter},
        "per_algorithm": per_alg,
        "e2e": {"value": e2e, "unit": "GTEPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": args.e2e_steps, "pipelined": True,
                "serial_value": (e2e_edges / e2e_serial_s / 1e9 * (world if world > 1 else 1)
                                 if e2e_serial_s > 0 else None)},
        "gpu_launches": int(launches),
        "clocks": clock_info,
        "tuning": tune_info,
    }
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    if cpu_leg:
        line["cpu_baseline"] = reference_cpu_baseline(args.cpu_sample_scale)
    g.close()
    if not args.no_batched:
        if world > 1:
            # the batch split over the ranks (every rank takes the same collective steps)
            line["sharded"] = sharded_section(args.batched_scale, torch, mg, tune=not args.no_tune)
        else:
            try:
                line["batched"] = batched_section(args.batched_scale, torch, mg, tune=not args.no_tune)
            except Exception as e:
                line["batched"] = {"unavailable": f"{type(e).__name__}: {e}"}
    adj_keep = {}
    if not args.no_extra:
        for key, fn in (("lattice", lambda t, m_: lattice_section(t, m_)),
                        ("pagerank_adjoint", lambda t, m_: adjoint_section(t, m_, keep=adj_keep))):
            try:
                line[key] = fn(torch, mg)
            except Exception as e:
                line[key] = {"unavailable": f"{type(e).__name__}: {e}"}
    if cpu_leg:
        # CPU baseline leg, after every timed region: the PageRank results checked
        # against the FP64 oracle (the error stated per run)
        try:
            chk = pagerank_fp64_check(h, x_pr, pr_last_iters, fixed_point=True)
            per_alg["pagerank"].update({k: chk[k] for k in ("l1_vs_fp64", "l1_vs_fp64_fixed_point")})
            line["cpu_baseline"]["pagerank_check"] = chk
        except Exception as e:
            per_alg["pagerank"]["l1_vs_fp64"] = f"unavailable: {type(e).__name__}: {e}"
        if adj_keep and isinstance(line.get("pagerank_adjoint"), dict) and "forward" in line["pagerank_adjoint"]:
            try:
                hk = adj_keep["h"]
                chk = pagerank_fp64_check(hk, adj_keep["x"], adj_keep["iterations"], weights=hk.weights_f32,
                                          fixed_point=False)
                line["pagerank_adjoint"]["forward"]["l1_vs_fp64"] = chk["l1_vs_fp64"]
                line["cpu_baseline"]["pagerank_adjoint_check"] = chk
            except Exception as e:
                line["pagerank_adjoint"]["forward"]["l1_vs_fp64"] = f"unavailable: {type(e).__name__}: {e}"
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
