"""The BFS / SSSP / CC / PageRank command-line drivers (the reference's
Algorithms/*/ mains: -g graph.mtx, -s sources, -o output, -p "name=value",
-c parameter file), run on the reference's small regression graphs written back
out as Matrix Market files from the golden fixtures."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from mirrorofmapgraph_b200 import _build

INT_MAX = 2**31 - 1
REF_SSSP_UNREACHED = 100000000  # Algorithms/SSSP/sssp.cu:139


@pytest.fixture(scope="module")
def bins():
    return {os.path.basename(p): p for p in _build.build_cli()}


def _write_mtx(path, d):
    ro, ci, vals = d["row_offsets"], d["col_idx"], d["values"]
    n = len(ro) - 1
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate integer general\n")
        f.write(f"{n} {n} {len(ci)}\n")
        for r in range(n):
            for k in range(ro[r], ro[r + 1]):
                f.write(f"{r + 1} {ci[k] + 1} {vals[k]}\n")


def _check_pagerank(x, d):
    # The reference's own pass test against CPUPR (relative L2 below its tol 0.1,
    # Algorithms/PageRank/PageRank.cu:316-321; CPUPR sweeps in place, so it is not a
    # tighter reference), then the FP64 restatement of the engine's schedule.
    ref = np.array(d["cpupr"])
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 0.1
    x64, _ = oracle.pr_refcompat(np.array(d["row_offsets"]), np.array(d["col_idx"]), 1)
    assert np.abs(x - x64).max() < 1.5e-5  # engine vs FP64 (as the library tests), six printed decimals


def _run(exe, *args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)


def _read(path, dtype):
    return np.loadtxt(path, dtype=dtype, ndmin=1)


def test_help_lists_the_reference_parameters(bins):
    for name in ("bfs", "sssp", "cc", "pagerank"):
        r = _run(bins[name], "-help")
        assert r.returncode == 1
        assert "-g <graph.mtx>" in r.stdout
        for p in ("iter_num", "max_queue_sizing", "device", "run_CPU"):
            assert p in r.stdout
    assert "origin" in _run(bins["bfs"], "-help").stdout
    assert "tol" in _run(bins["pagerank"], "-help").stdout


def test_missing_graph_prints_usage(bins):
    r = _run(bins["bfs"])
    assert r.returncode == 1 and "Usage" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
def test_drivers_match_reference_cpu_results(bins, mtx_fixtures, tmp_path, name):
    d = mtx_fixtures[name]
    g = str(tmp_path / f"{name}.mtx")
    _write_mtx(g, d)
    out = str(tmp_path / "out.txt")
    r = _run(bins["bfs"], "-g", g, "-o", out)
    assert r.returncode == 0, r.stderr
    assert _read(out, np.int64).tolist() == d["cpubfs_directed"]
    assert "Traversed edge:" in r.stdout
    r = _run(bins["sssp"], "-g", g, "-o", out)
    assert r.returncode == 0, r.stderr
    ref = [INT_MAX if x == REF_SSSP_UNREACHED else x for x in d["cpusssp_directed"]]
    assert _read(out, np.int64).tolist() == ref
    r = _run(bins["cc"], "-g", g, "-o", out)
    assert r.returncode == 0, r.stderr
    assert _read(out, np.int64).tolist() == d["cpucc"]
    r = _run(bins["pagerank"], "-g", g, "-o", out)
    assert r.returncode == 0, r.stderr
    x = _read(out, np.float64)
    _check_pagerank(x, d)
    if "cpubfs_undirected" in d:
        r = _run(bins["bfs"], "-g", g, "-o", out, "-p", "directed=0")
        assert r.returncode == 0, r.stderr
        assert _read(out, np.int64).tolist() == d["cpubfs_undirected"]
    # verbose=1 prints one line per level; the frontier sizes are the depth histogram
    r = _run(bins["bfs"], "-g", g, "-p", "verbose=1")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("iteration ")]
    depth = np.array(d["cpubfs_directed"])
    assert [int(ln.split("frontier ")[1].split(",")[0]) for ln in lines] == \
        np.bincount(depth[depth >= 0]).tolist()


@pytest.mark.gpu
def test_sources_file_and_parameter_file(bins, mtx_fixtures, tmp_path):
    d = mtx_fixtures["chesapeake"]
    g = str(tmp_path / "c.mtx")
    _write_mtx(g, d)
    srcf = tmp_path / "srcs.txt"
    srcf.write_text("3\n1\n")  # 1-based (origin=1): the last source run is vertex 0
    cfg = tmp_path / "params.cfg"
    cfg.write_text("directed=0\n")
    out = str(tmp_path / "out.txt")
    r = _run(bins["bfs"], "-g", g, "-s", str(srcf), "-c", str(cfg), "-o", out)
    assert r.returncode == 0, r.stderr
    assert "number of srcs used: 2" in r.stdout
    assert _read(out, np.int64).tolist() == d["cpubfs_undirected"]


@pytest.fixture(scope="module")
def shim_driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "shim_driver")
    here = os.path.dirname(os.path.abspath(__file__))
    r = subprocess.run(["g++", "-O1", "-std=c++17", "-I" + _build.INCLUDE, os.path.join(here, "cpp", "shim_driver.cpp"),
                        "-o", out, "-L" + _build.LIBDIR, "-lmapgraph_b200", "-Wl,-rpath," + _build.LIBDIR],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_cpp_shim_compiles_a_reference_style_driver(shim_driver):
    assert os.path.exists(shim_driver)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small", "chesapeake"])
def test_cpp_shim_results(shim_driver, mtx_fixtures, tmp_path, name):
    d = mtx_fixtures[name]
    g = str(tmp_path / f"{name}.mtx")
    _write_mtx(g, d)
    for prog, key in (("bfs", "cpubfs_directed"), ("sssp", "cpusssp_directed"), ("cc", "cpucc")):
        r = _run(shim_driver, prog, g, "0")
        assert r.returncode == 0, r.stderr
        got = [int(x) for x in r.stdout.split()]
        ref = [INT_MAX if (prog == "sssp" and x == REF_SSSP_UNREACHED) else x for x in d[key]]
        assert got == ref, prog
    r = _run(shim_driver, "pagerank", g, "0")
    assert r.returncode == 0, r.stderr
    x = np.array([float(v) for v in r.stdout.split()])
    _check_pagerank(x, d)
