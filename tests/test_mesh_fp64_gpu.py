"""FP64 end to end (ebg_mesh_signed_distance_f64): the CPU-runnable configuration -- the
20,480-triangle displaced icosphere, 4-wide SAH build, FP64 query points uniform in [-1.5,1.5]^3 --
against the reference's FP64 TriMeshSDF<double,short,4,4> on the same FP64 points.

Every query is re-evaluated with the reference's FP64 triangle test over the triangles within the
FP32 traversal's bound, so the distances are the reference's own: bit-identical except where two
triangles tie exactly (tolerance 1e-12 x diagonal there)."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12  # x diagonal


@pytest.fixture(scope="module")
def level5():
    v, f = W.displaced_icosphere(5, 1)
    ref = oracle.ref().mesh(v, f, kind=0, build=0, max_leaf_groups=4)
    return v, f, ref, TriMeshSDF(v, f, build="SAH")


def check_exact(d, d_ref, diag, what):
    assert d.dtype == np.float64, what
    err = np.abs(d - d_ref)
    assert err.max() <= TOL * diag, f"{what}: max err {err.max():.3e}"
    same = np.mean(d == d_ref)
    assert same > 0.9999, f"{what}: only {same:.6f} bit-identical"


def test_uniform_points_match_reference_fp64(level5):
    v, f, ref, m = level5
    p = np.random.default_rng(3).uniform(-1.5, 1.5, size=(300000, 3))
    d_ref = ref.sdf(p)
    d = m.signed_distance(torch.from_numpy(p).cuda()).cpu().numpy()
    torch.cuda.synchronize()
    m.check_status()
    check_exact(d, d_ref, m.diagonal, "uniform")


def test_near_surface_and_far_points_fp64(level5):
    v, f, ref, m = level5
    rng = np.random.default_rng(4)
    near = W.band_points(v, f, 50000, 5, 1e-3).astype(np.float64) + rng.uniform(-1e-7, 1e-7, (50000, 3))
    far = rng.uniform(-1e3, 1e3, size=(20000, 3))  # the FP32 rounding of these moves them ~1e-5
    for name, p in (("near", near), ("far", far)):
        d = m.signed_distance(torch.from_numpy(np.ascontiguousarray(p)).cuda()).cpu().numpy()
        check_exact(d, ref.sdf(p), m.diagonal, name)


def test_host_entry_and_value_are_fp64(level5):
    v, f, ref, m = level5
    p = np.random.default_rng(6).uniform(-1.5, 1.5, size=(4000, 3))
    d_ref = ref.sdf(p)
    d_host, tri = m.signed_distance(p, closest_tri=np.empty(4000, np.int32))
    check_exact(d_host, d_ref, m.diagonal, "host")
    assert tri.min() >= 0 and tri.max() < f.shape[0]
    for i in range(0, 4000, 211):
        assert m.value(p[i]) == pytest.approx(d_ref[i], abs=TOL * m.diagonal)


def test_mesh_far_from_the_origin():
    """A level-4 mesh moved about 60 diagonals from the origin, where FP32 rounds coordinates to
    about 1.5e-5 (4 x 1e-6 of the diagonal).  The FP32 pass's error bounds scale with the
    coordinates' magnitude there (fp32ErrorScale), so the FP64 entry point still returns the
    reference's FP64 values, and the FP32 entry point stays within 1e-6 of that magnitude with the
    reference's signs outside its band."""
    v, f = W.displaced_icosphere(4, 61)
    off = np.array([150.0, -120.0, 90.0])
    v = v + off
    rng = np.random.default_rng(62)
    p = np.concatenate([rng.uniform(-1.5, 1.5, size=(100000, 3)) + off, W.band_points(v, f, 20000, 63)])
    p = p.astype(np.float32).astype(np.float64)  # points the FP32 entry point can take exactly
    ref = oracle.ref().mesh(v, f, kind=0, build=0, max_leaf_groups=4)
    d_ref = ref.sdf(p)
    m = TriMeshSDF(v, f, build="SAH")
    scale = max(m.diagonal, float(np.abs(v).max()))
    d64 = m.signed_distance(torch.from_numpy(p).cuda()).cpu().numpy()
    check_exact(d64, d_ref, m.diagonal, "far mesh, FP64")
    d32 = m.signed_distance(torch.from_numpy(p.astype(np.float32)).cuda()).cpu().numpy().astype(np.float64)
    assert np.abs(d32 - d_ref).max() <= 1e-6 * scale
    out = np.abs(d_ref) > 1e-4 * scale
    assert np.sum(np.sign(d32[out]) != np.sign(d_ref[out])) == 0
