"""k-NN result checks shared by the point-cloud tests.

Distances must match exactly.  Indices must match exactly where the answer is unique; where equal
distances make several index lists correct (the reference orders ties by its visiting order, this
library by lowest index), each reported index must be a distinct point at exactly the reported
squared distance, computed with the reference's float arithmetic ((dx*dx + dy*dy) + dz*dz).
"""
import numpy as np


def d2_of(points, q, idx):
    """The reference's float squared distance from q to points[idx]."""
    d = (points[idx] - q).astype(np.float32)
    return (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]


def assert_knn_equiv(points, queries, idx_a, d2_a, idx_b, d2_b, self_ids=None):
    """(idx_a, d2_a) and (idx_b, d2_b) are both correct k-NN answers for the same queries.
    queries: (nq,3) float32, or None for self queries of self_ids (default every point)."""
    points = np.asarray(points, np.float32)
    idx_a = np.asarray(idx_a, np.int64)
    idx_b = np.asarray(idx_b, np.int64)
    assert np.array_equal(np.asarray(d2_a), np.asarray(d2_b)), "squared distances differ"
    if queries is None:
        ids = np.arange(points.shape[0]) if self_ids is None else np.asarray(self_ids)
        q = points[ids]
    else:
        q = np.asarray(queries, np.float32)
    differ = np.nonzero(np.any(idx_a != idx_b, axis=1))[0]
    for r in differ:
        for idx, d2 in ((idx_a[r], d2_a[r]), (idx_b[r], d2_b[r])):
            found = idx >= 0
            assert len(set(idx[found].tolist())) == found.sum(), f"row {r}: repeated index"
            if queries is None:
                assert not np.any(idx[found] == ids[r]), f"row {r}: self not excluded"
            assert np.array_equal(d2_of(points, q[r], idx[found]), np.asarray(d2)[found]), f"row {r}: wrong distance"
        # rows may only differ among equal distances
        da = np.asarray(d2_a[r])
        for j in np.nonzero(idx_a[r] != idx_b[r])[0]:
            assert np.count_nonzero(da == da[j]) > 1 or j == len(da) - 1, f"row {r}: index differs at a unique distance"
