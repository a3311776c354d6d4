"""Parity of the CUDA k-nearest-neighbour path (PointCloudBVH) with the oracle.

Contract: int32 neighbour indices bit-identical to the oracle's, ordered by (squared distance,
index) so ties resolve to the lowest index; squared distances bit-identical (the reference's
float arithmetic)."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, PointCloudBVH
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def knn_gpu(cloud, q, k, **kw):
    idx, d2 = cloud.knn(torch.from_numpy(np.ascontiguousarray(q, np.float32)).cuda(), k, **kw)
    torch.cuda.synchronize()
    cloud.check_status()
    return idx.cpu().numpy(), d2.cpu().numpy()


def test_reference_cloud_fixture(golden):
    g = golden("cloud2000.npz")
    c = PointCloudBVH(g["points"])
    for k, key, dkey in ((1, "lex1", "lexd1"), (8, "lex8", "lexd8")):
        idx, d2 = knn_gpu(c, g["queries"], k)
        assert np.array_equal(idx, g[key].astype(np.int32))
        assert np.array_equal(d2, g[dkey])
    # the reference's own closestPoints(k=5): same distances (its tie order follows its traversal)
    idx, d2 = knn_gpu(c, g["queries"], 5)
    assert np.array_equal(d2, g["d5"])
    # querying at a cloud point returns that point at distance 0 (TestPointCloudBVH.cpp:85-93)
    for i in range(0, 2000, 137):
        j, dd = c.closestPoint(g["points"][i])
        assert j == i and dd == 0.0


@pytest.mark.parametrize("balanced", [False, True])
@pytest.mark.parametrize("k", [1, 2, 3, 8, 17, 32])
@pytest.mark.parametrize("leaf", [1, 7, 16, 32])
def test_against_brute_force(k, leaf, balanced):
    pts = W.point_cloud(20000, 3)
    q = np.concatenate([W.uniform_points(3000, 4, 0, 1), pts[:500]])  # includes exact hits
    ref_idx, ref_d2 = oracle.port().knn_brute(pts, q, k)
    c = PointCloudBVH(pts, leaf_size=leaf, balanced=balanced)
    assert c.tree_info()["radix"] == (not balanced)
    idx, d2 = knn_gpu(c, q, k)
    assert np.array_equal(idx, ref_idx)
    assert np.array_equal(d2, ref_d2)
    idx2, d22 = knn_gpu(c, q, k, sort=False)
    assert np.array_equal(idx2, ref_idx) and np.array_equal(d22, ref_d2)


def test_ties_lowest_index():
    # duplicated points: every query ties between copies; the lowest index must win
    base = W.uniform_points(500, 7, 0, 1)
    pts = np.concatenate([base, base, base])
    q = W.uniform_points(1000, 8, 0, 1)
    ref_idx, ref_d2 = oracle.port().knn_brute(pts, q, 8)
    idx, d2 = knn_gpu(PointCloudBVH(pts), q, 8)
    assert np.array_equal(idx, ref_idx) and np.array_equal(d2, ref_d2)
    assert np.all(idx[:, 0] < 500)
    # grid points: many exactly equal distances
    g = W.grid_points(16, 0, 1)
    qq = W.grid_points(8, 0, 1)
    ref_idx, _ = oracle.port().knn_brute(g, qq, 8)
    idx, _ = knn_gpu(PointCloudBVH(g), qq, 8)
    assert np.array_equal(idx, ref_idx)


def test_tree_shapes():
    """The radix tree divides where the Morton curve jumps: leaves of at most leaf_size points, a
    depth the traversal stack holds, and far fewer nodes than points; a cloud of at most leaf_size
    points is one leaf."""
    pts = W.point_cloud(200000, 21)
    for leaf in (1, 8, 16, 32):
        info = PointCloudBVH(pts, leaf_size=leaf).tree_info()
        assert info["radix"] and 1 <= info["depth"] <= 31
        assert info["nodes"] <= max(1, len(pts) // max(1, leaf // 4))
    bal = PointCloudBVH(pts, leaf_size=16, balanced=True).tree_info()
    assert not bal["radix"] and bal["nodes"] == sum(-(-len(pts) // (16 * 4 ** j)) for j in range(1, bal["depth"] + 1))
    one = PointCloudBVH(pts[:16], leaf_size=16).tree_info()
    assert one["depth"] == 0


@pytest.mark.parametrize("leaf", [1, 16])
def test_degenerate_clouds(leaf):
    """Inputs whose Morton keys say little: one point repeated (every key equal: middle splits), points
    on a line at geometric spacing (most keys equal, a few far apart), two far clusters.  The answers
    are brute force's, lowest index first on ties."""
    rng = np.random.default_rng(22)
    same = np.tile(np.array([[0.25, 0.5, 0.75]], np.float32), (3000, 1))
    line = np.zeros((120, 3), np.float32)
    line[:, 0] = np.float32(2.0) ** -np.arange(120, dtype=np.float32)
    far = np.concatenate([rng.random((2000, 3), dtype=np.float32) * 1e-3,
                          1e4 + rng.random((2000, 3), dtype=np.float32)]).astype(np.float32)
    for pts, q in ((same, W.uniform_points(500, 23, 0, 1)),
                   (line, np.concatenate([line[::7], W.uniform_points(200, 24, -0.5, 1.5)])),
                   (far, np.concatenate([far[::50], W.uniform_points(200, 25, -1, 2)]))):
        c = PointCloudBVH(pts, leaf_size=leaf)
        info = c.tree_info()
        assert info["depth"] <= 31
        for k in (1, 8):
            ref_idx, ref_d2 = oracle.port().knn_brute(pts, q, k)
            idx, d2 = knn_gpu(c, q, k)
            assert np.array_equal(idx, ref_idx) and np.array_equal(d2, ref_d2)


def test_small_and_edge_cases():
    one = np.array([[0.5, 0.5, 0.5]], np.float32)
    c = PointCloudBVH(one)
    idx, d2 = knn_gpu(c, W.uniform_points(40, 1, 0, 1), 3)
    assert np.all(idx[:, 0] == 0) and np.all(idx[:, 1:] == -1) and np.all(np.isinf(d2[:, 1:]))
    with pytest.raises(EbgError):
        PointCloudBVH(np.zeros((0, 3), np.float32))
    with pytest.raises(EbgError):
        c.knn(torch.zeros((4, 3), device="cuda"), 33)
    idx, d2 = c.knn(np.zeros((0, 3), np.float32), 2)
    assert idx.shape == (0, 2)


def test_device_build_and_host_query_agree():
    pts = W.point_cloud(50000, 9)
    q = W.uniform_points(5000, 10, 0, 1)
    a = PointCloudBVH(torch.from_numpy(pts).cuda())
    b = PointCloudBVH(pts)
    ia, da = knn_gpu(a, q, 8)
    ib, db = b.knn(q, 8)
    assert np.array_equal(ia, ib) and np.array_equal(da, db)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle library not built")
def test_full_size_cloud_against_reference_sample():
    """16M-point cloud of the benchmark configuration: a 20k-query sample against the reference's
    own PointCloudBVH traversal (lexicographic state), k = 1 and 8, bit-exact."""
    pts = W.point_cloud(16 * 1024 * 1024, 1)
    q = W.uniform_points(20000, 2, 0, 1)
    c = PointCloudBVH(torch.from_numpy(pts).cuda())
    R = oracle.ref()
    rc = R.cloud(pts)
    for k in (1, 8):
        idx, d2 = knn_gpu(c, q, k)
        ri, rd = rc.knn(q, k, lex=True)
        assert np.array_equal(d2, rd)
        assert np.mean(idx == ri) > 0.9999  # the reference traversal's own ties at equal box distance


# --- self queries: allNearestNeighbors / nearestNeighbors ------------------------------------------
def test_self_knn_reference_fixture(golden):
    """The reference's own allNearestNeighbors on its test cloud (k = 1, 5) and the (d2, index)
    ordered traversal (k = 8): bit-identical."""
    g = golden("cloud2000.npz")
    c = PointCloudBVH(g["points"])
    for k, idx_key, d2_key in ((1, "self1", "selfd1"), (5, "self5", "selfd5"), (8, "selflex8", "selflexd8")):
        idx, d2 = c.all_nearest_neighbors(k)
        assert np.array_equal(d2, g[d2_key]), k
        assert np.array_equal(idx, g[idx_key].astype(np.int32)), k


@pytest.mark.parametrize("k", [1, 4, 16])
def test_self_knn_against_brute_force_with_duplicates(k):
    rng = np.random.default_rng(5)
    p = rng.uniform(0, 1, size=(12000, 3)).astype(np.float32)
    p[6000:6500] = p[:500]                         # exact duplicates: neighbours at d2 = 0
    p[7000:7200] = np.round(p[7000:7200] * 8) / 8  # lattice points: many equal distances
    c = PointCloudBVH(p, leaf_size=8)
    idx, d2 = c.all_nearest_neighbors(k)
    bi, bd = oracle.port().knn_brute_self(p, k)
    assert np.array_equal(d2, bd)
    assert np.array_equal(idx, bi)
    assert not np.any(idx == np.arange(p.shape[0])[:, None])  # never itself


def test_self_knn_points_subset_and_errors():
    rng = np.random.default_rng(6)
    p = rng.uniform(-1, 1, size=(30000, 3)).astype(np.float32)
    c = PointCloudBVH(p)
    all_idx, all_d2 = c.all_nearest_neighbors(3)
    ids = rng.integers(0, p.shape[0], size=5000)
    ids[:10] = ids[10]                               # repeated ids are fine
    idx, d2 = c.nearest_neighbors(ids, 3)
    assert np.array_equal(idx, all_idx[ids]) and np.array_equal(d2, all_d2[ids])
    i1, dd1 = c.nearestNeighbor(123)
    assert i1 == all_idx[123, 0] and dd1 == all_d2[123, 0]
    with pytest.raises(EbgError):
        c.nearest_neighbors([0, p.shape[0]], 1)
    # a one-point cloud has no other point
    one = PointCloudBVH(p[:1])
    idx1, d21 = one.all_nearest_neighbors(2)
    assert np.all(idx1 == -1) and np.all(np.isinf(d21))
