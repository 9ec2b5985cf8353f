"""The compat GASengine headers (include/compat): vertex programs written against
MapGraph's Program contract run through EnactorVertexCentric.

* Programs of this repository (tests/cpp/gas_user_programs.cu) exercise the
  generic kernels: label propagation (expand + contract + post_apply) against the
  connected-components oracle, and a gather sweep (gather_edge / gather_sum /
  apply) against a NumPy sum.
* MapGraph's own bfs / sssp / cc / pagerank programs, compiled unchanged from the
  reference tree into oracle/_ref (oracle/build_ref.sh), run with the tuned
  dispatch and on the generic kernels, against the reference's CPU results."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import mirrorofmapgraph_b200 as mg
from mirrorofmapgraph_b200 import _build

pytestmark = pytest.mark.gpu

INT_MAX = 2**31 - 1
REF_SSSP_UNREACHED = 100000000  # Algorithms/SSSP/sssp.cu:139
HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(os.path.dirname(HERE), "oracle", "_ref")


def _write_mtx(path, ro, ci, vals=None):
    n = len(ro) - 1
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate integer general\n")
        f.write(f"{n} {n} {len(ci)}\n")
        for r in range(n):
            for k in range(ro[r], ro[r + 1]):
                f.write(f"{r + 1} {ci[k] + 1} {1 if vals is None else vals[k]}\n")


@pytest.fixture(scope="module")
def user_driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("gas") / "gas_user_programs")
    nvcc = os.path.join(_build.CUDA_HOME, "bin", "nvcc")
    r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                        "-I" + os.path.join(_build.INCLUDE, "compat"), "-I" + _build.INCLUDE,
                        os.path.join(HERE, "cpp", "gas_user_programs.cu"), "-o", exe, "-L" + _build.LIBDIR,
                        "-lmapgraph_b200", "-Xlinker", "-rpath", "-Xlinker", _build.LIBDIR],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout.split()


@pytest.mark.parametrize("sym", [True, False])
def test_user_label_propagation_is_cc(user_driver, tmp_path, sym):
    h = mg.gen_rmat(12, 4, 21, symmetrize=sym)
    g = str(tmp_path / "g.mtx")
    _write_mtx(g, h.row_offsets, h.col_idx)
    got = np.array(_run(user_driver, "minlabel", g, 0), dtype=np.int64)
    np.testing.assert_array_equal(got, oracle.cc(h.row_offsets, h.col_idx))


def test_user_gather_sweep(user_driver, tmp_path):
    h = mg.gen_rmat(13, 16, 22, symmetrize=False)  # hubs above the lane-serial bound too
    g = str(tmp_path / "g.mtx")
    _write_mtx(g, h.row_offsets, h.col_idx)
    got = np.array(_run(user_driver, "insum", g, 1), dtype=np.int64)
    rows = np.repeat(np.arange(h.n), np.diff(h.row_offsets))
    ref = np.zeros(h.n, dtype=np.int64)
    np.add.at(ref, h.col_idx, rows + 1)
    np.testing.assert_array_equal(got, ref)


def _ref_run(exe, tmp_path, *args):
    out = str(tmp_path / "values.txt")
    _run(exe, *args, out)
    return np.loadtxt(out, ndmin=1)


def _ref_bins():
    bins = {m: os.path.join(REF_BIN, f"gas_ref_{m}") for m in ("tuned", "generic")}
    if not all(os.path.exists(b) for b in bins.values()):
        pytest.skip("oracle/_ref/gas_ref_* not built (needs the reference tree at build time)")
    return bins


@pytest.mark.parametrize("mode", ["tuned", "generic"])
@pytest.mark.parametrize("name", ["small", "trivialGraph", "chesapeake"])
def test_reference_programs_on_fixtures(mtx_fixtures, tmp_path, mode, name):
    exe = _ref_bins()[mode]
    d = mtx_fixtures[name]
    g = str(tmp_path / f"{name}.mtx")
    _write_mtx(g, d["row_offsets"], d["col_idx"], d["values"])
    assert _ref_run(exe, tmp_path, "bfs", g, 0, 1).astype(np.int64).tolist() == d["cpubfs_directed"]
    ref = [INT_MAX if x == REF_SSSP_UNREACHED else x for x in d["cpusssp_directed"]]
    assert _ref_run(exe, tmp_path, "sssp", g, 0, 1).astype(np.int64).tolist() == ref
    assert _ref_run(exe, tmp_path, "cc", g, 0, 0).astype(np.int64).tolist() == d["cpucc"]
    x = _ref_run(exe, tmp_path, "pagerank", g, 0, 1)
    cpu = np.array(d["cpupr"])
    assert np.linalg.norm(x - cpu) / np.linalg.norm(cpu) < 0.1  # the reference's own PR check
    x64, _ = oracle.pr_refcompat(np.array(d["row_offsets"]), np.array(d["col_idx"]), 1)
    assert np.abs(x - x64).max() < 1e-4
    if "cpubfs_undirected" in d:
        assert _ref_run(exe, tmp_path, "bfs", g, 0, 0).astype(np.int64).tolist() == d["cpubfs_undirected"]


@pytest.mark.parametrize("mode", ["tuned", "generic"])
def test_reference_programs_on_rmat(tmp_path, mode):
    exe = _ref_bins()[mode]
    h = mg.gen_rmat(11, 8, 23, symmetrize=False, weights="int", p0=1, p1=64)
    g = str(tmp_path / "r.mtx")
    _write_mtx(g, h.row_offsets, h.col_idx, h.weights_i32)
    np.testing.assert_array_equal(_ref_run(exe, tmp_path, "bfs", g, 3, 1).astype(np.int64),
                                  oracle.bfs(h.row_offsets, h.col_idx, [3]))
    np.testing.assert_array_equal(_ref_run(exe, tmp_path, "sssp", g, 3, 1).astype(np.int64),
                                  oracle.sssp(h.row_offsets, h.col_idx, h.weights_i32, [3]))
    np.testing.assert_array_equal(_ref_run(exe, tmp_path, "cc", g, 0, 0).astype(np.int64),
                                  oracle.cc(h.row_offsets, h.col_idx))
