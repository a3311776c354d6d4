"""MeshSDF and FlatMeshSDF (the reference's DCEL-face signed distance) on the GPU against the
reference's own values: the committed fixtures (made by the reference's MeshSDF<double,short,4> and
FlatMeshSDF<double,short>) and the reference library on larger meshes.  FP64 end to end, so the
bar is bit-identity (1e-12 x diagonal where two faces tie exactly)."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, FlatMeshSDF, MeshSDF, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12  # x diagonal


def check_exact(d, d_ref, diag, what, min_same=0.9999):
    assert d.dtype == np.float64, what
    err = np.abs(d - d_ref)
    assert err.max() <= TOL * diag, f"{what}: max err {err.max():.3e}"
    same = np.mean(d == d_ref)
    assert same >= min_same, f"{what}: only {same:.6f} bit-identical"


@pytest.mark.parametrize("name", ["dodecahedron.npz", "icosphere_l2.npz"])
def test_fixtures_bitexact(golden, name):
    g = golden(name)
    ms = MeshSDF(g["v"], g["f"], leaf_size=4)
    fl = FlatMeshSDF(g["v"], g["f"])
    check_exact(ms.signed_distance(g["p"]), g["dcel"], ms.diagonal, "MeshSDF", 1.0)
    check_exact(fl.signed_distance(g["p"]), g["flat"], fl.diagonal, "FlatMeshSDF", 1.0)
    # device entry points give the same numbers
    pd = torch.from_numpy(np.ascontiguousarray(g["p"])).cuda()
    assert np.array_equal(ms.signed_distance(pd).cpu().numpy(), g["dcel"])
    assert np.array_equal(fl.signed_distance(pd).cpu().numpy(), g["flat"])
    # the two classes differ from TriMeshSDF only in the last bits, as in the reference
    assert np.max(np.abs(g["dcel"] - g["ref"])) <= 1e-12 * ms.diagonal


@pytest.mark.parametrize("build", ["SAH", "Morton"])
def test_level4_against_reference(build):
    v, f = W.displaced_icosphere(4, 17)
    R = oracle.ref()
    ref_ms = R.mesh(v, f, kind=3, build=0)
    rng = np.random.default_rng(18)
    p = np.concatenate([rng.uniform(-1.5, 1.5, size=(60000, 3)),
                        W.band_points(v, f, 20000, 19, 1e-3).astype(np.float64)])
    d_ref = ref_ms.sdf(p, dcel=True)
    ms = MeshSDF(v, f, build=build)
    check_exact(ms.signed_distance(torch.from_numpy(p).cuda()).cpu().numpy(), d_ref, ms.diagonal, f"MeshSDF {build}")
    # FlatMeshSDF on a subset (every triangle for every point) with the winning faces
    fl = FlatMeshSDF(v, f, build=build)
    sub = p[::20]
    d_flat, tri = fl.signed_distance(sub, closest_tri=np.empty(sub.shape[0], np.int32))
    check_exact(d_flat, ref_ms.sdf(sub, flat=True), fl.diagonal, "FlatMeshSDF")
    _, tri_port = oracle.port().mesh_sdf_flat(v, f, sub)
    assert np.array_equal(tri, tri_port.astype(np.int32))


def test_value_and_non_finite():
    v, f = W.displaced_icosphere(2, 3)
    ms, fl, tm = MeshSDF(v, f), FlatMeshSDF(v, f), TriMeshSDF(v, f)
    for q in ([0.1, 0.2, 0.3], [1.4, -0.2, 0.05], [0.0, 0.0, 1.0]):
        a, b, c = ms.value(q), fl.value(q), tm.value(q)
        assert a == b
        assert abs(a - c) <= 1e-12 * tm.diagonal
    # a non-finite point is an invalid argument, as for the other entry points
    for sdf in (fl, ms):
        with pytest.raises(EbgError):
            sdf.signed_distance(np.array([[np.nan, 0.0, 0.0], [0.2, 0.0, 0.0]]))
    assert np.isfinite(fl.signed_distance(np.array([[0.2, 0.0, 0.0]]))[0])
