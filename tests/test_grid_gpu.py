"""Parity of the CUDA uniform-grid k-nearest-neighbour path (PointCloudHashGrid) with the oracle.

Contract: the same as PointCloudBVH's -- int32 indices in (squared distance, index) order, ties to
the lowest index, squared distances bit-identical to the reference's float arithmetic -- so the
grid's answers equal the brute-force oracle's and the BVH cloud's exactly.  Against the
reference's own grid (golden fixtures) the distances are identical and the indices equal up to the
order of equal distances (the reference orders ties by its visiting order)."""
import numpy as np
import pytest
import torch

import oracle
from _knn import assert_knn_equiv
from ebgeometry_b200 import EbgError, PointCloudBVH, PointCloudHashGrid
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def knn_gpu(obj, q, k):
    idx, d2 = obj.knn(torch.from_numpy(np.ascontiguousarray(q, np.float32)).cuda(), k)
    torch.cuda.synchronize()
    obj.check_status()
    return idx.cpu().numpy(), d2.cpu().numpy()


def test_reference_grid_fixture(golden):
    g = golden("grid2000.npz")
    grid = PointCloudHashGrid(g["points"])
    port = oracle.port()
    for k, ik, dk in ((1, "idx1", "d1"), (8, "idx8", "d8")):
        idx, d2 = knn_gpu(grid, g["queries"], k)
        assert_knn_equiv(g["points"], g["queries"], g[ik], g[dk], idx, d2)
        bi, bd = port.knn_brute(g["points"], g["queries"], k)
        assert np.array_equal(idx, bi) and np.array_equal(d2, bd)
    for k, ik, dk in ((1, "self1", "selfd1"), (5, "self5", "selfd5")):
        idx, d2 = grid.all_nearest_neighbors(k)
        assert_knn_equiv(g["points"], None, g[ik], g[dk], idx, d2)
        bi, bd = port.knn_brute_self(g["points"], k)
        assert np.array_equal(idx, bi) and np.array_equal(d2, bd)
    # querying at a cloud point returns that point at distance 0
    for i in range(0, 2000, 137):
        j, dd = grid.closestPoint(g["points"][i])
        assert j == i and dd == 0.0


def test_reference_edge_clouds(golden):
    """The reference test's edge cases: planar cloud, cluster plus a far outlier, coincident points,
    tiny and huge cell-size targets."""
    g = golden("grid2000.npz")
    port = oracle.port()
    for cloud, ik, dk, target in (("planar", "planar1", "planard1", 1.0), ("outlier", "outlier1", "outlierd1", 1.0),
                                  ("coincident", "coincident1", "coincidentd1", 1.0),
                                  ("c800", "tiny1", "tinyd1", 1e-6), ("c800", "huge1", "huged1", 1000.0)):
        grid = PointCloudHashGrid(g[cloud], target_per_cell=target)
        idx, d2 = grid.all_nearest_neighbors(1)
        assert_knn_equiv(g[cloud], None, g[ik], g[dk], idx, d2)
        bi, bd = port.knn_brute_self(g[cloud], 1)
        assert np.array_equal(idx, bi) and np.array_equal(d2, bd), cloud
        cells, _ = grid.grid_info()
        assert np.prod(cells) <= 64 + 8 * g[cloud].shape[0]


def test_small_clouds():
    empty = PointCloudHashGrid(np.zeros((0, 3), np.float32))
    assert empty.numPoints() == 0
    assert empty.closestPoint([0, 0, 0]) == (-1, float("inf"))
    assert empty.closestPoints([0, 0, 0], 4) == []
    idx, d2 = empty.all_nearest_neighbors(1)
    assert idx.shape == (0, 1)
    one = PointCloudHashGrid(np.array([[0.25, 0.5, 0.75]], np.float32))
    assert one.closestPoint([0.25, 0.5, 0.75]) == (0, 0.0)
    assert one.nearestNeighbor(0) == (-1, float("inf"))
    three = PointCloudHashGrid(W.uniform_points(3, 8, 0, 1))
    assert len(three.closestPoints([0.5, 0.5, 0.5], 10)) == 3


@pytest.mark.parametrize("k", [1, 3, 8, 17, 32])
@pytest.mark.parametrize("target", [0.3, 1.0, 4.0])
def test_against_brute_force(k, target):
    pts = W.point_cloud(20000, 3)
    q = np.concatenate([W.uniform_points(3000, 4, -0.2, 1.2), pts[:500]])  # outside the box, exact hits
    ref_idx, ref_d2 = oracle.port().knn_brute(pts, q, k)
    grid = PointCloudHashGrid(pts, target_per_cell=target)
    idx, d2 = knn_gpu(grid, q, k)
    assert np.array_equal(idx, ref_idx)
    assert np.array_equal(d2, ref_d2)
    hi, hd = grid.knn(q, k)  # host-array call
    assert np.array_equal(hi, ref_idx) and np.array_equal(hd, ref_d2)
    si, sd = grid.all_nearest_neighbors(k)
    bi, bd = oracle.port().knn_brute_self(pts, k)
    assert np.array_equal(si, bi) and np.array_equal(sd, bd)


def test_ties_lowest_index():
    base = W.uniform_points(500, 7, 0, 1)
    pts = np.concatenate([base, base, base])
    q = W.uniform_points(1000, 8, 0, 1)
    ref_idx, ref_d2 = oracle.port().knn_brute(pts, q, 8)
    idx, d2 = knn_gpu(PointCloudHashGrid(pts), q, 8)
    assert np.array_equal(idx, ref_idx) and np.array_equal(d2, ref_d2)
    si, sd = PointCloudHashGrid(pts).all_nearest_neighbors(4)
    bi, bd = oracle.port().knn_brute_self(pts, 4)
    assert np.array_equal(si, bi) and np.array_equal(sd, bd)


def test_equals_bvh_cloud_large():
    """A million-point clustered cloud: the grid and the BVH cloud give identical answers (the
    same contract), for external queries and for the self queries of a subset."""
    rng = np.random.default_rng(11)
    centres = rng.uniform(0, 1, (64, 3))
    pts = (centres[rng.integers(0, 64, 1_000_000)] + rng.normal(0, 0.02, (1_000_000, 3))).astype(np.float32)
    q = rng.uniform(-0.1, 1.1, (200_000, 3)).astype(np.float32)
    grid = PointCloudHashGrid(pts)
    bvh = PointCloudBVH(pts)
    for k in (1, 8):
        gi, gd = knn_gpu(grid, q, k)
        bi, bd = knn_gpu(bvh, q, k)
        assert np.array_equal(gi, bi) and np.array_equal(gd, bd)
    ids = rng.integers(0, pts.shape[0], 50_000)
    gi, gd = grid.nearest_neighbors(ids, 4)
    bi, bd = bvh.nearest_neighbors(ids, 4)
    assert np.array_equal(gi, bi) and np.array_equal(gd, bd)


def test_self_points_and_device_output():
    pts = W.point_cloud(5000, 21)
    grid = PointCloudHashGrid(pts)
    all_i, all_d = grid.all_nearest_neighbors(6)
    di, dd = grid.all_nearest_neighbors(6, device=True)
    torch.cuda.synchronize()
    assert np.array_equal(di.cpu().numpy(), all_i) and np.array_equal(dd.cpu().numpy(), all_d)
    ids = np.array([4999, 0, 17, 17, 2500])
    si, sd = grid.nearest_neighbors(ids, 6)
    assert np.array_equal(si, all_i[ids]) and np.array_equal(sd, all_d[ids])


def test_errors():
    pts = W.point_cloud(1000, 5)
    grid = PointCloudHashGrid(pts)
    with pytest.raises(EbgError):
        grid.nearest_neighbors([0, 1000], 1)
    with pytest.raises(EbgError):
        grid.knn(np.array([[np.nan, 0, 0]], np.float32), 1)
    with pytest.raises(EbgError):
        grid.knn(pts[:10], 33)
    with pytest.raises(EbgError):
        PointCloudHashGrid(np.array([[0, 0, np.inf]], np.float32))
    # the grid stays usable after reported errors
    idx, d2 = grid.knn(pts[:10], 1)
    assert np.array_equal(idx[:, 0], np.arange(10)) and np.all(d2 == 0)
