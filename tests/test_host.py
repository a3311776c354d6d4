"""Host-side logic without a GPU: the C ABI library loads and exports every symbol the header
declares, the host pseudonormals are bit-identical to the reference's DCEL, and the seeded
workloads have the properties the benchmarks assume."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from ebgeometry_b200 import _capi
from ebgeometry_b200 import workloads as W


def header_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"\b(ebg_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    names = header_functions()
    assert "ebg_mesh_signed_distance" in names
    lib = C.CDLL(_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table covers them all
    assert set(names) <= set(_capi.SIGNATURES), set(names) - set(_capi.SIGNATURES)


def _host_normals(v, f):
    v = np.ascontiguousarray(v, np.float64)
    f = np.ascontiguousarray(f, np.int32)
    t = f.shape[0]
    fn, vn, en = np.empty((t, 3)), np.empty((t, 3, 3)), np.empty((t, 3, 3))
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = _capi.lib.ebg_compute_pseudonormals(p(v), v.shape[0], p(f), t, p(fn), p(vn), p(en))
    return rc, fn, vn, en


@pytest.mark.parametrize("name", ["dodecahedron.npz", "icosphere_l2.npz"])
def test_pseudonormals_bitexact_vs_reference(golden, name):
    g = golden(name)
    rc, fn, vn, en = _host_normals(g["v"], g["f"])
    assert rc == 0
    assert np.array_equal(fn, g["face_n"])
    assert np.array_equal(vn, g["vert_n"])
    assert np.array_equal(en, g["edge_n"])


def test_pseudonormals_reject_bad_input():
    v = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0.0]])
    rc, *_ = _host_normals(v, np.array([[0, 1, 2]]))
    assert rc == 1 and b"degenerate" in _capi.lib.ebg_last_error()
    rc, *_ = _host_normals(v, np.array([[0, 1, 5]]))
    assert rc == 1 and b"out of range" in _capi.lib.ebg_last_error()


@pytest.mark.parametrize("level", [0, 1, 3])
def test_icosphere_watertight_outward(level):
    v, f = W.displaced_icosphere(level, 3)
    assert f.shape[0] == 20 * 4 ** level
    assert v.shape[0] == 10 * 4 ** level + 2
    e = np.sort(np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]]), axis=1)
    _, cnt = np.unique(e, axis=0, return_counts=True)
    assert np.all(cnt == 2)
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    assert np.all(np.einsum("ij,ij->i", np.cross(b - a, c - a), a + b + c) > 0)
    r = np.linalg.norm(v, axis=1)
    assert r.min() >= 0.92 - 1e-12 and r.max() <= 1.08 + 1e-12


def test_workloads_deterministic():
    assert np.array_equal(W.uniform_points(100, 1), W.uniform_points(100, 1))
    v, f = W.displaced_icosphere(2, 9)
    assert np.array_equal(W.band_points(v, f, 50, 4), W.band_points(v, f, 50, 4))
    g = W.grid_points(4, -1, 1)
    assert g.shape == (64, 3) and np.allclose(g[1] - g[0], [0.5, 0, 0])
    pc = W.point_cloud(1000, 2)
    assert pc.dtype == np.float32 and pc.min() >= 0 and pc.max() <= 1


def test_sample_points_are_the_references():
    """Random::samplePoints<double> (RandomImplem.hpp:27-44) through the library, against the
    reference's own (oracle/_ref) for a few seeds and sizes."""
    import oracle
    from ebgeometry_b200 import sample_points
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built (oracle/_ref)")
    for n, seed in ((1, 0), (1000, 20260708), (4096, 99)):
        assert np.array_equal(sample_points(n, seed), oracle.ref().sample_points(n, seed))
    assert sample_points(0, 5).shape == (0, 3)
