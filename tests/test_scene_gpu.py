"""Parity of the CUDA CSG union (BVHUnionIF over SphereSDF and Translate(Rotate(TriMeshSDF))) with
the reference: values within 1e-6 x the scene diagonal, signs identical where the reference value
is outside the +-1e-4 x diagonal band."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import BVHUnion, EbgError, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def scene_diag(spheres, meshes, poses):
    pts = [spheres[:, :3] - spheres[:, 3:4], spheres[:, :3] + spheres[:, 3:4]]
    for (v, _), ps in zip(meshes, poses):
        pts.append(W.rotate_points(v, -ps[0], int(ps[1])) + ps[2:5])
    allp = np.concatenate(pts)
    return float(np.linalg.norm(allp.max(0) - allp.min(0)))


def check(d, ref, diag, what):
    d = np.asarray(d, np.float64)
    assert np.all(np.isfinite(d)), what
    err = np.abs(d - ref).max()
    assert err <= 1e-6 * diag, f"{what}: {err:.3e} > {1e-6 * diag:.3e}"
    out = np.abs(ref) > 1e-4 * diag
    assert np.all(np.sign(d[out]) == np.sign(ref[out])), what


def test_reference_union_fixture(golden):
    g = golden("csg_small.npz")
    vo = np.concatenate([[0], np.cumsum(g["mesh_vcnt"])])
    fo = np.concatenate([[0], np.cumsum(g["mesh_fcnt"])])
    meshes = [(g["mesh_v"][vo[i]:vo[i + 1]], g["mesh_f"][fo[i]:fo[i + 1]]) for i in range(len(g["mesh_vcnt"]))]
    tms = [TriMeshSDF(v, f) for v, f in meshes]
    sc = BVHUnion(g["spheres"], tms, g["poses"])
    assert sc.num_objects() == len(g["spheres"]) + len(tms)
    diag = scene_diag(g["spheres"], meshes, g["poses"])
    d = sc.values(torch.from_numpy(g["p"].astype(np.float32)).cuda()).cpu().numpy()
    sc.check_status()
    check(d, g["ref"], diag, "BVHUnion fixture")
    check(sc.values(g["p"].astype(np.float32)), g["ref"], diag, "host entry")


@pytest.mark.parametrize("leaf", [1, 3, 8])
def test_random_scene_against_brute_force(leaf):
    sc = W.csg_scene(5, n_spheres=300, n_meshes=12, levels=(1, 4), mesh_radius=(0.05, 0.2))
    tms = [TriMeshSDF(v, f) for v, f in sc["meshes"]]
    u = BVHUnion(sc["spheres"], tms, sc["poses"], leaf_size=leaf)
    p = W.uniform_points(4000, 6, -1.3, 1.3)
    ref = oracle.port().scene_brute(sc["spheres"], sc["meshes"], sc["poses"], p.astype(np.float64))
    d = u.values(torch.from_numpy(p).cuda()).cpu().numpy()
    u.check_status()
    check(d, ref, scene_diag(sc["spheres"], sc["meshes"], sc["poses"]), f"leaf {leaf}")
    d2 = u.values(torch.from_numpy(p).cuda(), sort=False).cpu().numpy()
    check(d2, ref, scene_diag(sc["spheres"], sc["meshes"], sc["poses"]), "unsorted")


def test_spheres_only_and_meshes_only():
    rng = np.random.default_rng(1)
    sp = np.concatenate([rng.uniform(-1, 1, (50, 3)), rng.uniform(0.01, 0.2, (50, 1))], 1)
    p = W.uniform_points(2000, 2, -1.2, 1.2)
    ref = oracle.port().scene_brute(sp, [], np.zeros((0, 5)), p.astype(np.float64))
    d = BVHUnion(sp).values(p)
    check(d, ref, 3.0, "spheres")
    v, f = W.displaced_icosphere(3, 4, radius=0.5)
    poses = np.array([[30.0, 2, 0.2, 0.0, 0.1], [200.0, 0, -0.4, 0.3, 0.0]])
    ref = oracle.port().scene_brute(np.zeros((0, 4)), [(v, f), (v, f)], poses, p.astype(np.float64))
    m = TriMeshSDF(v, f)
    d = BVHUnion(None, [m, m], poses).values(p)  # one mesh instanced twice
    check(d, ref, 3.0, "meshes")
    assert np.any(d < 0)  # some points are inside


def test_scene_errors():
    with pytest.raises(EbgError):
        BVHUnion(np.zeros((0, 4)))
    v, f = W.displaced_icosphere(1, 1)
    with pytest.raises(EbgError):
        BVHUnion(None, [TriMeshSDF(v, f)], np.array([[10.0, 3, 0, 0, 0]]))


def test_batched_union_in_a_cuda_graph():
    """Many query batches of uneven length go in as one concatenated array, one persistent launch;
    the call issues only stream-ordered work, so it is captured once and replayed."""
    sc = W.csg_scene(7, n_spheres=200, n_meshes=8, levels=(1, 3), mesh_radius=(0.05, 0.2))
    tms = [TriMeshSDF(v, f) for v, f in sc["meshes"]]
    u = BVHUnion(sc["spheres"], tms, sc["poses"])
    rng = np.random.default_rng(8)
    lens = np.exp(rng.uniform(np.log(100), np.log(20000), size=40)).astype(int)
    p = np.concatenate([W.uniform_points(int(k), 100 + i, -1.2, 1.2) for i, k in enumerate(lens)])
    ref = u.values(torch.from_numpy(p).cuda()).cpu().numpy()
    pd = torch.from_numpy(p).cuda()
    out = torch.empty(p.shape[0], device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            u.values(pd, out=out, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        u.values(pd, out=out, stream=s)
    out.zero_()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)
