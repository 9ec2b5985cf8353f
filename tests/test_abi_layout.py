"""The ctypes mirror of the C ABI matches the header's struct layouts: a small C
program compiled against include/mapgraph_b200.h prints sizeof / offsetof of
every field of every public struct, and the ctypes structures must agree (CPU;
a mismatch would silently corrupt options and counters at the boundary)."""
import ctypes as C
import os
import subprocess

import pytest

from mirrorofmapgraph_b200 import _build
from mirrorofmapgraph_b200 import _lib as L

STRUCTS = {
    "mg_opts": L.MgOpts,
    "mg_stats": L.MgStats,
    "mg_pr_opts": L.MgPrOpts,
    "mg_part_level": L.MgPartLevel,
    "mg_level_record": L.MgLevelRecord,
    "mg_host_csr": L.MgHostCsr,
    "mg_tuning": L.MgTuning,
}


def _c_layout(tmp_path):
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "mapgraph_b200.h"',
             '#include "mapgraph_b200_io.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c11", "-I" + _build.INCLUDE, str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail("layout probe did not compile:\n" + r.stderr)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.splitlines():
        parts = line.split()
        got[tuple(parts[:-1])] = int(parts[-1])
    return got


def test_ctypes_structs_match_the_header(tmp_path):
    got = _c_layout(tmp_path)
    for cname, cls in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
