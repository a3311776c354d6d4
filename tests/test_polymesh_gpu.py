"""MeshSDF and FlatMeshSDF over polygon faces on the GPU (ebg_polymesh_*) against the reference's
own values: the committed fixtures (the reference's MeshSDF<double,short,4> and FlatMeshSDF over
soupToDCEL of the same soups) and the reference library on larger meshes.  FP64 end to end, so the
bar is bit-identity (1e-12 x diagonal where two faces tie exactly)."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, MeshSDF, PolygonFlatMeshSDF, PolygonMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12  # x diagonal


def check_exact(d, d_ref, diag, what, min_same=0.9999):
    assert d.dtype == np.float64, what
    err = np.abs(d - d_ref)
    assert err.max() <= TOL * diag, f"{what}: max err {err.max():.3e}"
    same = np.mean(d == d_ref)
    assert same >= min_same, f"{what}: only {same:.6f} bit-identical"


def near_points(v, off, idx, fn, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for f in rng.integers(0, off.size - 1, n):
        cv = v[idx[off[f]:off[f + 1]]]
        out.append(rng.dirichlet(np.ones(len(cv))) @ cv + rng.uniform(-1e-3, 1e-3) * fn[f])
    return np.array(out)


@pytest.mark.parametrize("name", ["prism", "quad", "mixed"])
@pytest.mark.parametrize("build", ["SAH", "Morton"])
def test_fixtures(golden, name, build):
    g = golden("polygons.npz")
    faces = (g[f"{name}_off"], g[f"{name}_idx"])
    m = PolygonMeshSDF(g[f"{name}_v"], faces, build=build)
    fn, c, vn, en = m.normals()
    assert np.array_equal(fn, g[f"{name}_face_n"]) and np.array_equal(c, g[f"{name}_centroid"])
    assert np.array_equal(vn, g[f"{name}_vert_n"]) and np.array_equal(en, g[f"{name}_edge_n"])
    p = g[f"{name}_p"]
    check_exact(m.signed_distance(p), g[f"{name}_ref"], m.diagonal, f"{name} MeshSDF")
    pd = torch.from_numpy(p).cuda()
    d = m.signed_distance(pd)
    torch.cuda.synchronize()
    m.check_status()
    check_exact(d.cpu().numpy(), g[f"{name}_ref"], m.diagonal, f"{name} MeshSDF device")
    flat = PolygonFlatMeshSDF(g[f"{name}_v"], faces)
    assert np.array_equal(flat.signed_distance(p), g[f"{name}_flat"])


@pytest.mark.parametrize("mesh", ["quad64", "mixed32", "prism40"])
def test_larger_meshes_against_reference(mesh):
    v, (off, idx) = {"quad64": lambda: W.displaced_quad_sphere(64, 7), "mixed32": lambda: W.mixed_polygon_sphere(32, 9),
                     "prism40": lambda: W.polygon_prism(40, 0.8, 1.5)}[mesh]()
    R = oracle.ref()
    ref = R.polymesh(v, off, idx)
    fn = ref.polygon_normals()[0]
    p = np.concatenate([W.uniform_points(20000, 3).astype(np.float64), near_points(v, off, idx, fn, 5000, 4)])
    m = PolygonMeshSDF(v, (off, idx))
    check_exact(m.signed_distance(p), ref.sdf(p, dcel=True), m.diagonal, mesh)
    # the brute force on a subset (every face for every point)
    sub = p[::25]
    face = np.empty(sub.shape[0], np.int32)
    df, face = PolygonFlatMeshSDF(v, (off, idx)).signed_distance(sub, closest_face=face)
    assert np.array_equal(df, ref.sdf(sub, flat=True))
    assert face.min() >= 0 and face.max() < off.size - 1


def test_triangle_soup_equals_triangle_meshsdf():
    """A triangle soup through the polygon path gives MeshSDF's triangle-mesh values exactly."""
    v, f = W.displaced_icosphere(4, 6)
    p = W.uniform_points(20000, 7).astype(np.float64)
    poly = PolygonMeshSDF(v, f)
    tri = MeshSDF(v, f, build="SAH")
    check_exact(poly.signed_distance(p), tri.signed_distance(p), poly.diagonal, "triangles")


def test_closest_face_and_from_file(tmp_path):
    v, (off, idx) = W.displaced_quad_sphere(8, 2)
    path = tmp_path / "q.obj"
    with open(path, "w") as fh:
        for q in v:
            fh.write(f"v {float(q[0])!r} {float(q[1])!r} {float(q[2])!r}\n")
        for k in range(off.size - 1):
            fh.write("f " + " ".join(str(int(i) + 1) for i in idx[off[k]:off[k + 1]]) + "\n")
    m = PolygonMeshSDF.from_file(path)
    ref_v, ref_off, ref_idx = oracle.ref().read_polysoup(path)
    ref = oracle.ref().polymesh(ref_v, ref_off, ref_idx)
    p = W.uniform_points(5000, 9).astype(np.float64)
    face = np.empty(p.shape[0], np.int32)
    d, face = m.signed_distance(p, closest_face=face)
    check_exact(d, ref.sdf(p, dcel=True), m.diagonal, "from file")
    assert face.min() >= 0 and face.max() < off.size - 1
    # FlatMeshSDF from the same file; its winner is the first face in soup order among those at the
    # smallest distance, MeshSDF's the lowest leaf position among equal |d| (faces around a shared
    # vertex tie exactly), so the two face indices need not agree, the values must
    fl = PolygonFlatMeshSDF.from_file(path)
    ff = np.empty(p.shape[0], np.int32)
    dfl, ff = fl.signed_distance(p, closest_face=ff)
    assert np.array_equal(dfl, ref.sdf(p, flat=True))
    assert ff.min() >= 0 and ff.max() < off.size - 1


def test_errors():
    v, faces = W.polygon_prism(6)
    m = PolygonMeshSDF(v, faces)
    with pytest.raises(EbgError):
        m.signed_distance(np.array([[np.nan, 0.0, 0.0]]))
    # usable afterwards
    assert np.isfinite(m.value([0.1, 0.2, 0.0]))
    with pytest.raises(EbgError):
        PolygonMeshSDF(v, [[0, 1, 2, 1]])  # a vertex twice in one face
    flat = v.copy()
    flat[:, 2] = 0.0
    with pytest.raises(EbgError):
        PolygonMeshSDF(flat, faces)
