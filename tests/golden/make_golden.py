"""Regenerates the golden fixtures in this directory from the reference's own CPU code.

Run from the repository root, in a checkout where the reference tree is present:

    python tests/golden/make_golden.py

Inputs: the reference's three bundled Matrix Market graphs (ingested by the
reference's own reader, b40c/graph/builder/market.cuh) and seeded synthetic graphs
from this package's generators. Outputs are the results of the reference functions
CPUBFS / CPUSSSP / CPUCC / CPUPR (built by oracle/build_ref.sh into
oracle/_ref/libmgref.so):

  mtx_fixtures.json   edge lists of small.mtx, trivialGraph.mtx, chesapeake.mtx as the
                      reference ingests them, with the reference results (directed, and
                      undirected BFS/SSSP for chesapeake)
  synthetic.npz       seeded ER (4,096 vertices / 65,536 edges, weights U{1..64}) and
                      R-MAT (scale 10, edge factor 16, symmetrised, weights U{1..255}):
                      a CSR checksum of each graph and the reference results
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
import mirrorofmapgraph_b200 as mg  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
MTX = ["small", "trivialGraph", "chesapeake"]

ER = dict(n=4096, m=65536, seed=20140601, wmax=64)
ER_SOURCES = [0, 1, 17, 4095]
RMAT = dict(scale=10, ef=16, seed=7, wmax=255)
RMAT_SOURCES = [0, 3, 100, 1023]


def csr_digest(ro, ci, w=None) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ro, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(ci, dtype=np.int32).tobytes())
    if w is not None:
        h.update(np.ascontiguousarray(w).tobytes())
    return h.hexdigest()


def er_graph():
    return mg.gen_er(ER["n"], ER["m"], ER["seed"], weights="int", p0=1, p1=ER["wmax"])


def rmat_graph():
    return mg.gen_rmat(RMAT["scale"], RMAT["ef"], RMAT["seed"], symmetrize=True, weights="int", p0=1,
                       p1=RMAT["wmax"])


def main() -> None:
    if not oracle.have_ref():
        raise SystemExit("reference tree not available: cannot regenerate golden fixtures")
    R = oracle.Ref
    fixtures = {}
    for name in MTX:
        path = os.path.join(oracle.REFERENCE_DIR, "smallRegressionGraphs", name + ".mtx")
        ro, ci, vals, co, ri = R.load_market(path)
        csc = (co, ri, None)
        d = {
            "n": int(ro.size - 1), "row_offsets": ro.tolist(), "col_idx": ci.tolist(), "values": vals.tolist(),
            "col_offsets": co.tolist(), "row_idx": ri.tolist(),
            "cpubfs_directed": R.bfs(ro, ci, 0, 1, csc)[0].tolist(),
            "cpusssp_directed": R.sssp(ro, ci, vals, 0, 1, csc)[0].tolist(),
            "cpucc": R.cc(ro, ci, csc)[0].tolist(),
            "cpupr": [float(x) for x in R.pr(ro, ci, csc)[0]],
        }
        if name == "chesapeake":
            d["cpubfs_undirected"] = R.bfs(ro, ci, 0, 0, csc)[0].tolist()
            # CPUSSSP with directed=0 reads CSR weights by CSC position
            # (sssp.cu:181-191); chesapeake has unit weights, so it is exact here.
            d["cpusssp_undirected"] = R.sssp(ro, ci, vals, 0, 0, csc)[0].tolist()
        fixtures[name] = d
    with open(os.path.join(HERE, "mtx_fixtures.json"), "w") as f:
        json.dump(fixtures, f, separators=(",", ":"))

    out = {}
    g = er_graph()
    out["er_digest"] = np.frombuffer(bytes.fromhex(csr_digest(g.row_offsets, g.col_idx, g.weights_i32)),
                                     dtype=np.uint8)
    out["er_sources"] = np.array(ER_SOURCES, dtype=np.int32)
    out["er_bfs"] = np.stack([R.bfs(g.row_offsets, g.col_idx, s, 1)[0] for s in ER_SOURCES])
    out["er_sssp"] = np.stack([R.sssp(g.row_offsets, g.col_idx, g.weights_i32, s, 1)[0] for s in ER_SOURCES])
    out["er_cc"] = R.cc(g.row_offsets, g.col_idx)[0]
    out["er_pr"] = R.pr(g.row_offsets, g.col_idx)[0]
    g = rmat_graph()
    out["rmat_digest"] = np.frombuffer(bytes.fromhex(csr_digest(g.row_offsets, g.col_idx, g.weights_i32)),
                                       dtype=np.uint8)
    out["rmat_sources"] = np.array(RMAT_SOURCES, dtype=np.int32)
    out["rmat_bfs"] = np.stack([R.bfs(g.row_offsets, g.col_idx, s, 1)[0] for s in RMAT_SOURCES])
    out["rmat_sssp"] = np.stack([R.sssp(g.row_offsets, g.col_idx, g.weights_i32, s, 1)[0] for s in RMAT_SOURCES])
    out["rmat_cc"] = R.cc(g.row_offsets, g.col_idx)[0]
    out["rmat_pr"] = R.pr(g.row_offsets, g.col_idx)[0]
    np.savez_compressed(os.path.join(HERE, "synthetic.npz"), **out)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
