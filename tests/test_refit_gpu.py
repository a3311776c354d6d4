"""Refitting a mesh to moved vertices (PackedBVH::refit for TriMeshSDF; ebg_mesh_refit).

Contract: after a refit the mesh answers exactly as the reference does for the moved vertices --
the parity contract of every mesh query (|d - d_ref| <= 1e-6 * diag; signs equal outside the
1e-4 * diag band), pseudonormals bit-identical to a fresh build of the moved soup -- while the
tree keeps its topology.  A refit to the same positions changes nothing, bit for bit."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, MeshSDF, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6
BAND = 1e-4


def check_parity(d_gpu, d_ref, diag, what=""):
    d_gpu = np.asarray(d_gpu, np.float64)
    err = np.abs(d_gpu - d_ref)
    assert np.all(np.isfinite(d_gpu)), what
    assert err.max() <= REL_TOL * diag, f"{what}: max err {err.max():.3e} > {REL_TOL * diag:.3e}"
    out = np.abs(d_ref) > BAND * diag
    assert np.sum(np.sign(d_gpu[out]) != np.sign(d_ref[out])) == 0, what


def sdf(mesh, p):
    tri = np.empty(p.shape[0], np.int32)
    return mesh.signed_distance(np.ascontiguousarray(p, np.float32), closest_tri=tri)


def check_exact(d, d_ref, diag, what):
    """FP64: the reference's own values (1e-12 x diagonal where two triangles tie exactly)."""
    assert np.max(np.abs(d - d_ref)) <= 1e-12 * diag, what
    assert np.mean(d == d_ref) > 0.9999, what


def rotate(v, deg, axis):
    t = np.deg2rad(deg)
    c, s = np.cos(t), np.sin(t)
    i, j = [(1, 2), (2, 0), (0, 1)][axis]
    out = v.copy()
    out[:, i] = c * v[:, i] - s * v[:, j]
    out[:, j] = s * v[:, i] + c * v[:, j]
    return out


@pytest.mark.parametrize("build,on_device", [("SAH", False), ("Morton", False), ("Morton", True)])
def test_refit_to_same_positions_changes_nothing(build, on_device):
    v, f = W.displaced_icosphere(4, 3)
    p = np.concatenate([W.uniform_points(20000, 4), W.band_points(v, f, 5000, 5)])
    m = TriMeshSDF(v, f, build=build, on_device=on_device)
    d0, t0 = sdf(m, p)
    n0 = m.normals()
    p64 = p.astype(np.float64)
    e0 = m.signed_distance(p64)
    m.refit(v)
    d1, t1 = sdf(m, p)
    assert np.array_equal(d0, d1) and np.array_equal(t0, t1)
    assert np.array_equal(e0, m.signed_distance(p64))
    for a, b in zip(n0, m.normals()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("build,on_device", [("SAH", False), ("Morton", True)])
def test_refit_moved_mesh_matches_reference(build, on_device):
    """Moved vertices: a different displacement field, then rotated, scaled and translated -- the
    boxes of every node change; results must be the reference's for the moved soup."""
    v, f = W.displaced_icosphere(4, 3)
    v2, f2 = W.displaced_icosphere(4, 9)
    assert np.array_equal(f, f2)
    v2 = rotate(v2 * 0.7, 33.0, 2) + np.array([0.3, -0.2, 0.1])
    p = np.concatenate([W.uniform_points(30000, 6), W.band_points(v2, f2, 10000, 7)])
    m = TriMeshSDF(v, f, build=build, on_device=on_device)
    m.refit(v2)
    fresh = TriMeshSDF(v2, f2, build=build, on_device=on_device)
    for a, b in zip(m.normals(), fresh.normals()):
        assert np.array_equal(a, b)
    assert m.info["lo"] == fresh.info["lo"] and m.info["hi"] == fresh.info["hi"]
    assert m.diagonal == fresh.diagonal
    d_ref = oracle.ref().mesh(v2, f2).sdf(p.astype(np.float64))
    d, _ = sdf(m, p)
    check_parity(d, d_ref, m.diagonal, "refit FP32 + band")
    # FP64 end to end and the DCEL-face evaluator read the refitted FP64 records
    check_exact(m.signed_distance(p.astype(np.float64)), d_ref, m.diagonal, "refit FP64")
    dref_dcel = oracle.ref().mesh(v2, f2, kind=3).sdf(p.astype(np.float64), dcel=True)
    md = MeshSDF(v, f, build=build)
    md.refit(v2)
    check_exact(md.signed_distance(p.astype(np.float64)), dref_dcel, m.diagonal, "refit DCEL")


def test_refit_device_tensor_and_repeated_motion():
    v, f = W.displaced_icosphere(3, 11)
    m = TriMeshSDF(v, f, build="Morton", on_device=True)
    p = W.uniform_points(20000, 12)
    R = oracle.ref()
    for step in range(4):
        vs = rotate(v, 10.0 * step, step % 3) * (1.0 + 0.1 * step) + 0.05 * step
        m.refit(torch.from_numpy(vs).cuda())
        d, _ = sdf(m, p)
        check_parity(d, R.mesh(vs, f).sdf(p.astype(np.float64)), m.diagonal, f"step {step}")


def test_refit_errors_leave_the_mesh_usable():
    v, f = W.displaced_icosphere(3, 13)
    m = TriMeshSDF(v, f)
    p = W.uniform_points(5000, 14)
    d0, _ = sdf(m, p)
    with pytest.raises(EbgError):
        m.refit(v[:-1])  # wrong vertex count
    bad = v.copy()
    bad[5, 1] = np.nan
    with pytest.raises(EbgError):
        m.refit(bad)
    flat = v.copy()
    a, b, c = f[0]
    flat[c] = flat[a]  # triangle 0 loses its area
    with pytest.raises(EbgError):
        m.refit(flat)
    d1, _ = sdf(m, p)
    assert np.array_equal(d0, d1)
