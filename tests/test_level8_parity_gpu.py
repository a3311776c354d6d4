"""Parity on the headline workload: the level-8 displaced icosphere (1,310,720 triangles, device
Morton build) queried on a seeded stratified sample of its 512^3 cell-centre grid over
[-1.25,1.25]^3 and its 16,777,216 near-surface points, plain and seeded (a trained model attached
as per-cell entry cuts), against the reference's TriMeshSDF<double,short,4,4> (oracle/_ref) on the
same points: |d - d_ref| <= 1e-6 x diagonal everywhere and identical signs outside the band
|d_ref| <= 1e-4 x diagonal (TriMeshSDF::signedDistance, MeshDistanceFunctionsImplem.hpp:480-509)."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import SeedModel, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

GRID, LO, HI = 512, -1.25, 1.25
N_BAND = 16 * 1024 * 1024
SAMPLE = 240_000


def _stratified_sample(rng):
    """Grid cell centres and band points in their workload proportion (134,217,728 : 16,777,216)."""
    n_grid = GRID ** 3
    ng = int(round(SAMPLE * n_grid / (n_grid + N_BAND)))
    gi = rng.choice(n_grid, size=ng, replace=False)
    h = (HI - LO) / GRID
    ix, iy, iz = gi % GRID, (gi // GRID) % GRID, gi // (GRID * GRID)
    grid = np.stack([LO + h * (ix + 0.5), LO + h * (iy + 0.5), LO + h * (iz + 0.5)], 1).astype(np.float32)
    return grid, SAMPLE - ng


@pytest.fixture(scope="module")
def level8():
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built (oracle/_ref)")
    v, f = W.displaced_icosphere(8, 1)
    rng = np.random.default_rng(2024)
    grid, nb = _stratified_sample(rng)
    band = W.band_points(v, f, N_BAND, 2, 1e-3)  # the workload's band points, then a sample of them
    p = np.concatenate([grid, band[rng.choice(N_BAND, size=nb, replace=False)]])
    mesh = TriMeshSDF(v, f, build="Morton", leaf_size=8, on_device=True)
    ref = oracle.ref().mesh(v, f, kind=0, build=1, max_leaf_groups=4)  # TriMeshSDF<double,short,4,4>, Morton
    d_ref = ref.sdf(p.astype(np.float64))
    return mesh, p, d_ref, v, f


def _check(mesh, d, d_ref):
    diag = mesh.diagonal
    d = np.asarray(d, np.float64)
    err = np.abs(d - d_ref)
    outside = np.abs(d_ref) > 1e-4 * diag
    mism = int(np.sum(np.sign(d[outside]) != np.sign(d_ref[outside])))
    assert err.max() <= 1e-6 * diag, (err.max(), 1e-6 * diag)
    assert mism == 0, mism
    return err.max()


def test_level8_plain_matches_reference(level8):
    mesh, p, d_ref, _, _ = level8
    d = mesh.signed_distance(torch.from_numpy(p).cuda()).cpu().numpy()
    mesh.check_status()
    print("level-8 plain max |d - d_ref| / diag:", _check(mesh, d, d_ref) / mesh.diagonal)


def test_level8_seeded_matches_reference_and_plain(level8):
    mesh, p, d_ref, _, _ = level8
    seed = SeedModel.train(mesh, num_samples=1 << 23, steps=600, batch=1 << 17, rng_seed=7, lo=[LO] * 3, hi=[HI] * 3)
    pts = torch.from_numpy(p).cuda()
    d_plain = mesh.signed_distance(pts)
    d_seed = mesh.signed_distance(pts, seed=seed)
    mesh.check_status()
    assert torch.equal(d_seed, d_plain)
    print("level-8 seeded max |d - d_ref| / diag:", _check(mesh, d_seed.cpu().numpy(), d_ref) / mesh.diagonal)
