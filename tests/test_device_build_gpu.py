"""The device (GPU) build of the Morton and the binned-SAH tree, records and oriented boxes: a mesh
built on the GPU answers exactly as the host-built one -- the same tree and leaf order, so the same
distances and closest triangles bit for bit -- and matches the reference."""
import time

import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, MeshSDF, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def query(m, p, **kw):
    pd = torch.from_numpy(np.ascontiguousarray(p)).cuda()
    tri = torch.empty(pd.shape[0], dtype=torch.int32, device="cuda")
    d, tri = m.signed_distance(pd, closest_tri=tri, **kw)
    torch.cuda.synchronize()
    m.check_status()
    return d.cpu().numpy(), tri.cpu().numpy()


@pytest.mark.parametrize("build", ["Morton", "SAH"])
@pytest.mark.parametrize("level,leaf", [(3, 8), (5, 8), (5, 1), (5, 32), (6, 8), (7, 4)])
def test_device_build_equals_host_build(level, leaf, build):
    v, f = W.displaced_icosphere(level, 3)
    p = np.concatenate([W.uniform_points(100000, 4), W.band_points(v, f, 30000, 5)])
    host = TriMeshSDF(v, f, build=build, leaf_size=leaf)
    dev = TriMeshSDF(v, f, build=build, leaf_size=leaf, on_device=True)
    assert dev.info["num_nodes"] == host.info["num_nodes"] and dev.info["num_leaves"] == host.info["num_leaves"]
    assert dev.info["depth"] == host.info["depth"]
    assert dev.info["num_triangles"] == f.shape[0]
    assert dev.info["leaf_size"] == leaf and dev.info["depth"] >= 2
    np.testing.assert_array_equal(dev.info["lo"], host.info["lo"])
    np.testing.assert_array_equal(dev.info["hi"], host.info["hi"])
    dh, th = query(host, p)
    dd, td = query(dev, p)
    assert np.array_equal(dh, dd)
    assert np.array_equal(th, td)
    # the FP64 path and the DCEL faces too
    p64 = p[:20000].astype(np.float64)
    assert np.array_equal(host.signed_distance(p64), dev.signed_distance(p64))


@pytest.mark.parametrize("level", [2, 6])
def test_device_pseudonormals_bitexact(level, golden):
    """The device build computes the pseudonormals on the GPU (the angle weights' acos on the host):
    bit-identical to the host restatement and so to the reference's DCEL."""
    v, f = W.displaced_icosphere(level, 12)
    host = TriMeshSDF(v, f, build="Morton")
    dev = TriMeshSDF(v, f, build="Morton", on_device=True)
    for a, b in zip(host.normals(), dev.normals()):
        assert np.array_equal(a, b)
    g = golden("icosphere_l2.npz")
    fn, vn, en = TriMeshSDF(g["v"], g["f"], build="Morton", on_device=True).normals()
    assert np.array_equal(fn, g["face_n"]) and np.array_equal(vn, g["vert_n"]) and np.array_equal(en, g["edge_n"])


def test_device_build_rejects_bad_soups():
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [2, 0, 0]], np.float64)
    with pytest.raises(EbgError):  # zero area
        TriMeshSDF(v, np.array([[0, 1, 3]]), build="Morton", on_device=True)
    v5 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1]], np.float64)
    with pytest.raises(EbgError):  # one edge (0,1) shared by three triangles
        TriMeshSDF(v5, np.array([[0, 1, 2], [1, 0, 3], [0, 1, 4]]), build="Morton", on_device=True)


def test_device_build_against_reference():
    v, f = W.displaced_icosphere(4, 8)
    p = W.uniform_points(50000, 9).astype(np.float64)
    m = TriMeshSDF(v, f, build="Morton", on_device=True)
    d_ref = oracle.ref().mesh(v, f, kind=0, build=1).sdf(p)
    d = m.signed_distance(p)
    assert np.max(np.abs(d - d_ref)) <= 1e-12 * m.diagonal
    ms = MeshSDF(v, f, build="Morton", on_device=True)
    d_dcel = oracle.ref().mesh(v, f, kind=3, build=1).sdf(p, dcel=True)
    assert np.max(np.abs(ms.signed_distance(p) - d_dcel)) <= 1e-12 * ms.diagonal


def test_device_build_small_and_errors():
    tv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    tf = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
    p = W.uniform_points(2000, 10, -2, 2)
    for build in ("Morton", "SAH"):
        for leaf in (8, 1, 2):
            host = TriMeshSDF(tv, tf, build=build, leaf_size=leaf)
            dev = TriMeshSDF(tv, tf, build=build, leaf_size=leaf, on_device=True)
            assert np.array_equal(query(host, p)[0], query(dev, p)[0]), (build, leaf)
    with pytest.raises(EbgError):
        TriMeshSDF(tv, tf, build="Morton", leaf_size=33, on_device=True)


def test_device_sah_build_identical_centroids():
    """Two coincident copies of a mesh (separate vertices): each triangle's copy has the same
    centroid, so at leaf size 1 some ranges have no SAH split; both builds halve them and agree."""
    v, f = W.displaced_icosphere(2, 1)
    v2 = np.concatenate([v, v])
    f2 = np.concatenate([f, f + v.shape[0]])
    p = W.uniform_points(20000, 4)
    for leaf in (1, 2, 4):
        host = TriMeshSDF(v2, f2, build="SAH", leaf_size=leaf)
        dev = TriMeshSDF(v2, f2, build="SAH", leaf_size=leaf, on_device=True)
        dh, th = query(host, p)
        dd, td = query(dev, p)
        assert np.array_equal(dh, dd) and np.array_equal(th, td), leaf


@pytest.mark.parametrize("build", ["Morton", "SAH"])
def test_level8_device_build_time(build):
    """The level-8 mesh (1,310,720 triangles) built both ways; reported, and equal on a sample."""
    v, f = W.displaced_icosphere(8, 1)
    t0 = time.time()
    host = TriMeshSDF(v, f, build=build)
    t1 = time.time()
    dev = TriMeshSDF(v, f, build=build, on_device=True)
    t2 = time.time()
    print(f"level-8 {build} build: host {t1 - t0:.3f} s, device {t2 - t1:.3f} s; "
          f"nodes {host.info['num_nodes']} / {dev.info['num_nodes']}, leaves {host.info['num_leaves']} / "
          f"{dev.info['num_leaves']}, depth {host.info['depth']} / {dev.info['depth']}")
    p = np.concatenate([W.grid_points(64, -1.25, 1.25), W.band_points(v, f, 100000, 11)])
    assert np.array_equal(query(host, p)[0], query(dev, p)[0])
