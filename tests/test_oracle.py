"""Pins the CPU oracle: the plain-C restatement (oracle/ebg_port.c) against the golden vectors the
reference produced (tests/golden/, made by tests/golden/make_golden.py) and against the reference's
own known answers (Tests/TestTriangle.cpp).  Runs without a GPU."""
import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module")
def port():
    return oracle.port()


def test_triangle_kats(port, golden):
    k = golden("triangle_kat.npz")
    for i in range(len(k["expected"])):
        fn = np.array([0, 0, 1.0])
        for scalar in (True, False):
            d = port.triangle_sd(k["v"][i], fn, k["vn"][i], k["en"][i], k["p"][i], scalar=scalar)
            assert d == pytest.approx(k["expected"][i], rel=1e-12, abs=1e-12)
        assert port.triangle_sd(k["v"][i], fn, k["vn"][i], k["en"][i], k["p"][i], scalar=True) == k["ref"][i]


def test_trisoa_min_over_lanes(port, golden):
    g = golden("trisoa.npz")
    fn = np.array([0, 0, 1.0])
    for ci, cnt in enumerate(g["counts"]):
        for qi, q in enumerate(g["p"]):
            best = np.inf
            for t in range(cnt):  # strict <: the first of equal |d| wins (TriangleSoAImplem.hpp:1171-1177)
                d = port.triangle_sd(g["tris"][t], fn, g["vn"][t], g["en"][t], q)
                if abs(d) < abs(best):
                    best = d
            assert best == g["ref"][ci, qi]


@pytest.mark.parametrize("name", ["dodecahedron.npz", "icosphere_l2.npz"])
def test_mesh_normals_and_sdf_bitexact(port, golden, name):
    g = golden(name)
    tn, vn, en = port.mesh_normals(g["v"], g["f"])
    assert np.array_equal(tn, g["face_n"])
    assert np.array_equal(vn, g["vert_n"])
    assert np.array_equal(en, g["edge_n"])
    d, _ = port.mesh_sdf_brute(g["v"], g["f"], g["p"])
    # brute force over the soup vs the reference's BVH traversal: same values, same order-free min
    assert np.max(np.abs(d - g["ref"])) <= 1e-12


@pytest.mark.parametrize("name", ["dodecahedron.npz", "icosphere_l2.npz"])
def test_dcel_face_port_bitexact(port, golden, name):
    """The DCEL face algorithm (MeshSDF / FlatMeshSDF) restated in C reproduces the reference's
    FlatMeshSDF and MeshSDF<double,short,4> values bit for bit (they differ from TriMeshSDF's
    TriangleSoA test in the last bits)."""
    g = golden(name)
    d, _ = port.mesh_sdf_flat(g["v"], g["f"], g["p"])
    assert np.array_equal(d, g["flat"])
    assert np.array_equal(d, g["dcel"])


def test_dodecahedron_flat_agrees(golden):
    g = golden("dodecahedron.npz")
    # the reference's own relational check (Tests/TestBVH.cpp:112-194, margin 1e-6 for double)
    assert np.max(np.abs(g["ref"] - g["flat"])) <= 1e-6


def test_knn_brute_matches_reference_traversal(port, golden):
    g = golden("cloud2000.npz")
    for k, key, dkey in ((1, "lex1", "lexd1"), (8, "lex8", "lexd8")):
        idx, d2 = port.knn_brute(g["points"], g["queries"], k)
        assert np.array_equal(idx, g[key].astype(np.int32))
        assert np.array_equal(d2, g[dkey])
    # the reference's own closestPoints agrees on distances (its ties follow traversal order)
    idx, d2 = port.knn_brute(g["points"], g["queries"], 5)
    assert np.array_equal(d2, g["d5"])


def test_csg_brute(port, golden):
    g = golden("csg_small.npz")
    vo = np.concatenate([[0], np.cumsum(g["mesh_vcnt"])])
    fo = np.concatenate([[0], np.cumsum(g["mesh_fcnt"])])
    meshes = [(g["mesh_v"][vo[i]:vo[i + 1]], g["mesh_f"][fo[i]:fo[i + 1]]) for i in range(len(g["mesh_vcnt"]))]
    out = port.scene_brute(g["spheres"], meshes, g["poses"], g["p"])
    assert np.max(np.abs(out - g["brute"])) <= 1e-12
    assert np.max(np.abs(out - g["ref"])) <= 1e-12


@pytest.mark.skipif(not oracle.ref_available(), reason="reference oracle library not built on this host")
def test_reference_reproduces_fixtures(golden):
    R = oracle.ref()
    g = golden("icosphere_l2.npz")
    m = R.mesh(g["v"], g["f"], kind=0, build=0, max_leaf_groups=4)
    assert np.array_equal(m.sdf(g["p"]), g["ref"])
    c = golden("cloud2000.npz")
    idx, d2 = R.cloud(c["points"]).knn(c["queries"], 8, lex=True)
    assert np.array_equal(idx, c["lex8"])


def test_self_knn_brute_matches_reference(port, golden):
    """The C restatement of the self queries (the point itself excluded, (d2, index) order) against
    the reference's allNearestNeighbors on its own test cloud."""
    g = golden("cloud2000.npz")
    for k, idx_key, d2_key in ((1, "self1", "selfd1"), (5, "self5", "selfd5"), (8, "selflex8", "selflexd8")):
        idx, d2 = port.knn_brute_self(g["points"], k)
        assert np.array_equal(d2, g[d2_key])
        assert np.array_equal(idx, g[idx_key].astype(np.int32))


def test_grid_fixture_brute(port, golden):
    """The reference's PointCloudHashGrid answers on its own test clouds equal brute force (the C
    restatement): distances exactly, indices up to the order of equal distances."""
    from _knn import assert_knn_equiv
    g = golden("grid2000.npz")
    for k, ik, dk in ((1, "idx1", "d1"), (8, "idx8", "d8")):
        idx, d2 = port.knn_brute(g["points"], g["queries"], k)
        assert_knn_equiv(g["points"], g["queries"], g[ik], g[dk], idx, d2)
    for k, ik, dk in ((1, "self1", "selfd1"), (5, "self5", "selfd5")):
        idx, d2 = port.knn_brute_self(g["points"], k)
        assert_knn_equiv(g["points"], None, g[ik], g[dk], idx, d2)
    for cloud, ik, dk in (("planar", "planar1", "planard1"), ("outlier", "outlier1", "outlierd1"),
                          ("coincident", "coincident1", "coincidentd1"), ("c800", "tiny1", "tinyd1"),
                          ("c800", "huge1", "huged1")):
        idx, d2 = port.knn_brute_self(g[cloud], 1)
        assert_knn_equiv(g[cloud], None, g[ik], g[dk], idx, d2)
