"""The Python binding's ctypes structures (ebgeometry_b200/_capi.py) against the C header
(include/ebgeometry_b200.h): a C program compiled against the header prints the size of every
option/report struct and the offset of each of its fields, and they must equal the ctypes layout,
field by field and in the same order.  A field added to one side only would otherwise shift every
later option silently.  The batch descriptor the Python union fills as an int64 (n, 3) array is
checked the same way."""
import ctypes
import os
import shutil
import subprocess

import pytest

from conftest import ROOT
from ebgeometry_b200 import _capi

CC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else shutil.which("gcc")

PAIRS = {
    "ebg_build_opts": _capi.BuildOpts,
    "ebg_phase_timings": _capi.PhaseTimings,
    "ebg_query_opts": _capi.QueryOpts,
    "ebg_seed_opts": _capi.SeedOpts,
    "ebg_seed_report": _capi.SeedReport,
    "ebg_mesh_info": _capi.MeshInfo,
    "ebg_query_stats": _capi.QueryStats,
    "ebg_attach_opts": _capi.AttachOpts,
    "ebg_attach_report": _capi.AttachReport,
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("abi")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "ebgeometry_b200.h"', "int main(void) {"]
    for cname, cls in PAIRS.items():
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append('  printf("ebg_batch sizeof %zu\\n", sizeof(ebg_batch));')
    for fname in ("points_dev", "n", "out_dev"):
        lines.append(f'  printf("ebg_batch {fname} %zu\\n", offsetof(ebg_batch, {fname}));')
    lines += ["  return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = str(d / "layout")
    r = subprocess.run([CC, "-std=c11", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    layout = {}
    for line in out.splitlines():
        s, f, v = line.split()
        layout[(s, f)] = int(v)
    return layout


@pytest.mark.parametrize("cname", sorted(PAIRS))
def test_ctypes_struct_matches_the_header(c_layout, cname):
    cls = PAIRS[cname]
    assert c_layout[(cname, "sizeof")] == ctypes.sizeof(cls), cname
    for fname, _ in cls._fields_:
        assert c_layout[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_batch_descriptor_is_three_int64_words(c_layout):
    # the Python union writes each descriptor as int64 (points, n, out)
    assert c_layout[("ebg_batch", "sizeof")] == 24
    assert [c_layout[("ebg_batch", f)] for f in ("points_dev", "n", "out_dev")] == [0, 8, 16]
