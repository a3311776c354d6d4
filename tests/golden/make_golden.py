"""Generates the committed golden fixtures of tests/golden/ from the reference itself.

Run where the reference sources exist (the directory is the first argument, or the
EBG_REFERENCE_DIR environment variable):

    python tests/golden/make_golden.py [REFERENCE]

It builds nothing but the oracle (``make -C oracle``) and writes small .npz files:

* ``triangle_kat.npz``   -- the known-answer cases of the reference's Tests/TestTriangle.cpp
  (right triangle (0,0,0),(4,0,0),(0,4,0) with the test's normals; expected 5, -3, 0, 1, sqrt(8)),
  with the reference's scalar Triangle::signedDistance output for each.
* ``trisoa.npz``         -- Tests/TestTriangleSoA.cpp's four disjoint triangles and six query
  points, with TriangleSoAT<double,4>::signedDistance outputs for 4, 2 and 1 packed triangles.
* ``dodecahedron.npz``   -- Tests/data/dodecahedron.obj read through the reference's parser, the
  ten query points of Tests/TestBVH.cpp plus 500 seeded points, and the reference's
  TriMeshSDF<double,short,4,4> (SAH) and FlatMeshSDF values and DCEL pseudonormals.
* ``icosphere_l2.npz``   -- a displaced level-2 icosphere with the reference's pseudonormals and
  TriMeshSDF values at 2000 seeded points (including 500 within 1e-3 of the surface).
* ``cloud2000.npz``      -- Tests/TestPointCloudBVH.cpp's 2000-point cloud (mt19937 seed 20260708),
  external queries and the self queries of allNearestNeighbors (k = 1, 5 and lexicographic k = 8)
  and 200 external queries (seed 99), with the reference's PointCloudBVH closestPoints (k = 1, 5)
  and the same traversal with (d2, index) ordering.
* ``grid2000.npz``       -- Tests/TestPointCloudHashGrid.cpp's clouds: the 2000-point cloud (seed
  20260708) with 200 external queries (seed 99), the reference's PointCloudHashGrid closestPoints
  (k = 1, 8) and allNearestNeighbors (k = 1, 5); its edge-case clouds (a planar cloud, a cluster with
  a distant outlier, 16 coincident points, cell-size targets 1e-6 and 1000) with allNearestNeighbors
  (k = 1).  Indices are the reference's own (ties in its visiting order).
* ``polygons.npz``       -- polygon meshes (a heptagonal prism, a displaced 4x4 quad sphere, a 6x6
  quad sphere with every other quad split into triangles) with the reference's DCEL normals
  (soupToDCEL) and its MeshSDF<double,short,4> (SAH) and FlatMeshSDF values at 1000 points each
  (uniform, plus points near the faces).
* ``csg_small.npz``      -- a union of 40 spheres and 3 posed displaced icospheres evaluated by the
  reference's BVHUnion over Translate(Rotate(TriMeshSDF)) and SphereSDF at 1000 points.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ebgeometry_b200 import workloads as W  # noqa: E402


def main(reference: str) -> None:
    oracle.build(reference)
    R = oracle.ref()

    # --- Triangle KATs (TestTriangle.cpp:37-113) ---------------------------------------------------
    v = np.array([[0, 0, 0], [4, 0, 0], [0, 4, 0]], np.float64)
    z = np.array([0, 0, 1.0])
    s2 = 1.0 / np.sqrt(2.0)
    cases = [  # (vertex normals, edge normals, point, expected)
        ([z, z, z], [z, z, z], [1, 1, 5], 5.0),
        ([z, z, z], [z, z, z], [1, 1, -3], -3.0),
        ([z, z, z], [z, z, z], [1, 1, 0], 0.0),
        ([z, z, z], [z, [s2, s2, 0], z], [2 + s2, 2 + s2, 0], 1.0),
        ([z, [s2, -s2, 0], z], [z, z, z], [6, -2, 0], np.sqrt(8.0)),
    ]
    kv, kvn, ken, kp, kexp, kref = [], [], [], [], [], []
    for vn, en, p, e in cases:
        vn, en, p = np.array(vn, np.float64), np.array(en, np.float64), np.array(p, np.float64)
        kv.append(v), kvn.append(vn), ken.append(en), kp.append(p), kexp.append(e)
        kref.append(R.triangle_sd(v, vn, en, p))
    np.savez(os.path.join(HERE, "triangle_kat.npz"), v=np.array(kv), vn=np.array(kvn), en=np.array(ken),
             p=np.array(kp), expected=np.array(kexp), ref=np.array(kref))

    # --- TriangleSoA (TestTriangleSoA.cpp:30-83) ---------------------------------------------------
    tris = np.array([[[3.0 * i, 0, 0], [3.0 * i + 1, 0, 0], [3.0 * i, 1, 0]] for i in range(4)])
    nrm = np.tile(np.array([0, 0, 1.0]), (4, 3, 1))  # Triangle's default normals are unset -> use +z
    qp = np.array([[0.25, 0.25, 0.1], [3.25, 0.25, -0.2], [6.25, 0.25, 0.05], [9.25, 0.25, 0], [-5, -5, -5],
                   [20, 20, 20]], np.float64)
    out = np.zeros((3, qp.shape[0]))
    for ci, cnt in enumerate((4, 2, 1)):
        for qi, q in enumerate(qp):
            out[ci, qi] = R.trisoa4_sd(tris[:cnt], nrm[:cnt], nrm[:cnt], q)
    np.savez(os.path.join(HERE, "trisoa.npz"), tris=tris, vn=nrm, en=nrm, p=qp, counts=np.array([4, 2, 1]), ref=out)

    # --- dodecahedron fixture (TestBVH.cpp:36-52, Tests/data/dodecahedron.obj) ------------------------
    dv, df = R.read_soup(os.path.join(reference, "Tests", "data", "dodecahedron.obj"))
    q10 = np.array([[0, 0, 0], [0.5, 0.5, 0.5], [1, 1, 1], [1.5, 0, 0], [0, 1.5, 0], [0, 0, 1.5], [-1.5, -1.5, -1.5],
                    [3, 3, 3], [10, 0, 0], [-5, 2, 1]], np.float64)
    qr = np.random.default_rng(11).uniform(-2.5, 2.5, (500, 3)).astype(np.float32).astype(np.float64)
    dq = np.concatenate([q10, qr])
    m = R.mesh(dv, df, kind=0, build=0, max_leaf_groups=4)
    fn, vn, en = m.normals()
    md = R.mesh(dv, df, kind=3, build=0)  # MeshSDF<double,short,4> over the DCEL faces
    np.savez(os.path.join(HERE, "dodecahedron.npz"), v=dv, f=df.astype(np.int32), p=dq, ref=m.sdf(dq),
             flat=m.sdf(dq, flat=True), dcel=md.sdf(dq, dcel=True), face_n=fn, vert_n=vn, edge_n=en)

    # --- displaced icosphere, level 2 ------------------------------------------------------------------
    iv, iff = W.displaced_icosphere(2, 1234)
    m = R.mesh(iv, iff, kind=0, build=0, max_leaf_groups=4)
    fn, vn, en = m.normals()
    qa = W.uniform_points(1500, 5, -1.5, 1.5).astype(np.float64)
    qb = W.band_points(iv, iff, 500, 6, 1e-3).astype(np.float64)
    iq = np.concatenate([qa, qb])
    md = R.mesh(iv, iff, kind=3, build=0)
    np.savez(os.path.join(HERE, "icosphere_l2.npz"), v=iv, f=iff, p=iq, ref=m.sdf(iq), flat=m.sdf(iq, flat=True),
             dcel=md.sdf(iq, dcel=True), face_n=fn, vert_n=vn, edge_n=en)

    # --- point cloud (TestPointCloudBVH.cpp:58-120) ----------------------------------------------------
    pts = R.make_cloud_mt19937(2000, 20260708)
    qs = R.make_cloud_mt19937(200, 99)
    c = R.cloud(pts)
    i1, d1 = c.knn(qs, 1, lex=False)
    i5, d5 = c.knn(qs, 5, lex=False)
    l1, e1 = c.knn(qs, 1, lex=True)
    l8, e8 = c.knn(qs, 8, lex=True)
    # self queries: the reference's allNearestNeighbors (itself excluded) and the lexicographic state
    s1, t1 = c.self_knn(1, lex=False)
    s5, t5 = c.self_knn(5, lex=False)
    sl8, tl8 = c.self_knn(8, lex=True)
    np.savez(os.path.join(HERE, "cloud2000.npz"), points=pts, queries=qs, idx1=i1, d1=d1, idx5=i5, d5=d5, lex1=l1,
             lexd1=e1, lex8=l8, lexd8=e8, self1=s1, selfd1=t1, self5=s5, selfd5=t5, selflex8=sl8, selflexd8=tl8)

    # --- uniform-grid cloud (TestPointCloudHashGrid.cpp:60-330) ----------------------------------------
    g = R.grid(pts)
    gi1, gd1 = g.knn(qs, 1)
    gi8, gd8 = g.knn(qs, 8)
    gs1, gt1 = g.all_nn(1)
    gs5, gt5 = g.all_nn(5)
    planar = R.make_cloud_mt19937(500, 7)
    planar[:, 2] = 0
    ps1, pt1 = R.grid(planar).all_nn(1)
    outl = np.concatenate([R.make_cloud_mt19937(999, 12), np.array([[1e6, 0.5, 0.5]], np.float32)])
    os1, ot1 = R.grid(outl).all_nn(1)
    coinc = np.tile(np.array([[1, 2, 3]], np.float32), (16, 1))
    cs1, ct1 = R.grid(coinc).all_nn(1)
    c800 = R.make_cloud_mt19937(800, 9)
    tiny1, tinyd1 = R.grid(c800, 1e-6).all_nn(1)
    huge1, huged1 = R.grid(c800, 1000.0).all_nn(1)
    np.savez(os.path.join(HERE, "grid2000.npz"), points=pts, queries=qs, idx1=gi1, d1=gd1, idx8=gi8, d8=gd8,
             self1=gs1, selfd1=gt1, self5=gs5, selfd5=gt5, planar=planar, planar1=ps1, planard1=pt1,
             outlier=outl, outlier1=os1, outlierd1=ot1, coincident=coinc, coincident1=cs1,
             coincidentd1=ct1, c800=c800, tiny1=tiny1, tinyd1=tinyd1, huge1=huge1, huged1=huged1)

    # --- polygon meshes (MeshSDF / FlatMeshSDF over DCEL polygon faces) --------------------------------
    out = {}
    for name, (pv, (off, idx)) in (("prism", W.polygon_prism(7)), ("quad", W.displaced_quad_sphere(4, 3)),
                                   ("mixed", W.mixed_polygon_sphere(6, 5))):
        rng = np.random.default_rng(len(name))
        pts = [rng.uniform(-1.6, 1.6, (700, 3))]
        # near the faces: a random convex combination of a face's vertices, moved along its normal
        pm = R.polymesh(pv, off, idx)
        fn, _, _, _ = pm.polygon_normals()
        fsel = rng.integers(0, off.size - 1, 300)
        near = []
        for f in fsel:
            cv = pv[idx[off[f]:off[f + 1]]]
            w = rng.dirichlet(np.ones(len(cv)))
            near.append(w @ cv + rng.uniform(-1e-3, 1e-3) * fn[f])
        pts.append(np.array(near))
        pq = np.concatenate(pts)
        fnn, cen, vn, en = pm.polygon_normals()
        out.update({f"{name}_v": pv, f"{name}_off": off, f"{name}_idx": idx, f"{name}_p": pq,
                    f"{name}_ref": pm.sdf(pq, dcel=True), f"{name}_flat": pm.sdf(pq, flat=True),
                    f"{name}_face_n": fnn, f"{name}_centroid": cen, f"{name}_vert_n": vn, f"{name}_edge_n": en})
    np.savez(os.path.join(HERE, "polygons.npz"), **out)

    # --- small CSG union --------------------------------------------------------------------------------
    sc = W.csg_scene(77, n_spheres=40, n_meshes=3, levels=(1, 3), mesh_radius=(0.15, 0.3))
    bb = []
    for (mv, _), pose in zip(sc["meshes"], sc["poses"]):
        # world position of a local vertex x: R^-1 x + t, the inverse of RotateIF's point map
        wv = W.rotate_points(mv, -pose[0], int(pose[1])) + pose[2:5]
        bb.append(np.concatenate([wv.min(0), wv.max(0)]))
    bb = np.array(bb)
    scene = R.scene(sc["spheres"], sc["meshes"], sc["poses"], bb)
    sq = np.random.default_rng(3).uniform(-1.3, 1.3, (1000, 3)).astype(np.float32).astype(np.float64)
    vals = scene.value(sq)
    brute = scene.value(sq, brute=True)
    mv_all = np.concatenate([mv for mv, _ in sc["meshes"]])
    mf_all = np.concatenate([mf for _, mf in sc["meshes"]])
    vcnt = np.array([mv.shape[0] for mv, _ in sc["meshes"]])
    fcnt = np.array([mf.shape[0] for _, mf in sc["meshes"]])
    np.savez(os.path.join(HERE, "csg_small.npz"), spheres=sc["spheres"], poses=sc["poses"], bboxes=bb,
             mesh_v=mv_all, mesh_f=mf_all, mesh_vcnt=vcnt, mesh_fcnt=fcnt, p=sq, ref=vals, brute=brute)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EBG_REFERENCE_DIR")
    if not ref_dir:
        sys.exit("usage: make_golden.py REFERENCE_DIR (or set EBG_REFERENCE_DIR)")
    main(ref_dir)
