import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
INT_MAX = 2**31 - 1


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a engine)")
    config.addinivalue_line("markers", "slow: larger graphs, minutes rather than seconds")


def _ensure_built():
    from mirrorofmapgraph_b200 import _build
    import oracle
    if not os.path.exists(_build.LIB):
        _build.build()
    oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def mtx_fixtures():
    with open(os.path.join(GOLDEN, "mtx_fixtures.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def synthetic_golden():
    return dict(np.load(os.path.join(GOLDEN, "synthetic.npz")))


def ref_sssp_to_engine(d):
    """The reference CPU check writes 100000000 for unreached vertices (sssp.cu:139);
    the engine uses INT_MAX (sssp.h:43)."""
    d = np.asarray(d, dtype=np.int64)
    return np.where(d == 100000000, INT_MAX, d).astype(np.int32)
