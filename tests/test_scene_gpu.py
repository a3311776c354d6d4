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


def _world_boxes(sc):
    """World AABB of every posed mesh (RotateIF applied backwards, then the translation)."""
    bb = []
    for (v, f), ps in zip(sc["meshes"], sc["poses"]):
        w = W.rotate_points(v, -ps[0], int(ps[1])) + ps[2:5]
        bb.append(np.concatenate([w.min(0) - 1e-9, w.max(0) + 1e-9]))
    return np.array(bb)


def _near_surface_points(sc, per_mesh, seed, width):
    """Points within +-width of each posed mesh's surface, in world coordinates."""
    pts = []
    for i, ((v, f), ps) in enumerate(zip(sc["meshes"], sc["poses"])):
        local = W.band_points(v, f, per_mesh, seed + i, width).astype(np.float64)
        pts.append(W.rotate_points(local, -ps[0], int(ps[1])) + ps[2:5])
    return np.concatenate(pts).astype(np.float32)


def test_batches_match_concatenated_and_replay_in_a_graph():
    """ebg_scene_eval_batches: many batches of uneven length (one of them empty) in one call give
    the concatenated call's values bit for bit, and the call is captured once and replayed."""
    sc = W.csg_scene(9, n_spheres=300, n_meshes=10, levels=(1, 3), mesh_radius=(0.05, 0.2))
    u = BVHUnion(sc["spheres"], [TriMeshSDF(v, f) for v, f in sc["meshes"]], sc["poses"])
    rng = np.random.default_rng(4)
    lens = list(np.exp(rng.uniform(np.log(50), np.log(30000), size=60)).astype(int)) + [0, 7]
    batches = [torch.from_numpy(W.uniform_points(int(k), 300 + i, -1.2, 1.2)).cuda() for i, k in enumerate(lens)]
    ref = u.values(torch.cat(batches)).cpu().numpy()
    outs = u.values_batches(batches)
    u.check_status()
    got = torch.cat(outs).cpu().numpy()
    assert np.array_equal(got, ref)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            u.values_batches(batches, outs=outs, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        u.values_batches(batches, outs=outs, stream=s)
    for o in outs:
        o.zero_()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(torch.cat(outs).cpu().numpy(), ref)


def test_batch_sizes_that_do_not_add_up_are_rejected():
    sc = W.csg_scene(9, n_spheres=20, n_meshes=0)
    u = BVHUnion(sc["spheres"])
    b = [torch.from_numpy(W.uniform_points(100, 1)).cuda()]
    outs = [torch.full((100,), 7.0, device="cuda")]
    import ctypes as C

    from ebgeometry_b200 import _capi
    desc = torch.tensor([[b[0].data_ptr(), 100, outs[0].data_ptr()]], dtype=torch.int64, device="cuda")
    opts = _capi.QueryOpts()
    # a total of 150 for batches of 100 points: nothing is computed, the status check reports it
    assert _capi.lib.ebg_scene_eval_batches(u._h, C.c_void_p(desc.data_ptr()), 1, 150, C.byref(opts), None) == 0
    with pytest.raises(EbgError):
        u.check_status()
    assert torch.all(outs[0] == 7.0)


def test_union_near_surface_points_take_the_fp64_pass():
    """Points within 1e-5 of the posed meshes' surfaces: the FP64 pass evaluates them as the
    reference's BVHUnionIF<double> does, so their signs agree inside the band as well."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built (oracle/_ref)")
    sc = W.csg_scene(13, n_spheres=200, n_meshes=12, levels=(2, 4), mesh_radius=(0.05, 0.2))
    u = BVHUnion(sc["spheres"], [TriMeshSDF(v, f) for v, f in sc["meshes"]], sc["poses"])
    p = _near_surface_points(sc, 3000, 50, 1e-5)
    ref = oracle.ref().scene(sc["spheres"], sc["meshes"], sc["poses"], _world_boxes(sc)).value(p.astype(np.float64))
    d = u.values(torch.from_numpy(p).cuda()).cpu().numpy().astype(np.float64)
    u.check_status()
    diag = scene_diag(sc["spheres"], sc["meshes"], sc["poses"])
    inband = np.abs(ref) <= 1e-4 * diag
    assert inband.mean() > 0.9
    # FP64 values, returned as float32
    assert np.all(np.abs(d[inband] - ref[inband]) <= 1e-7 * np.abs(ref[inband]) + 1e-12)
    clear = inband & (np.abs(ref) > 1e-12)
    assert np.all(np.sign(d[clear]) == np.sign(ref[clear]))
    d32 = u.values(torch.from_numpy(p).cuda(), fp64_band=False).cpu().numpy().astype(np.float64)
    check(d32, ref, diag, "FP32 only")  # within the tolerance even without the band pass
    assert np.abs(d32 - ref).max() > np.abs(d - ref).max()


def test_configuration_scene_sample_against_reference():
    """The batched union's configuration: 4,096 spheres and 256 displaced icospheres of levels 3-7
    (23.9 M triangles) at random poses; a seeded sample of uniform points in the scene box and of
    points within 1e-5 of the meshes' surfaces, in batches of uneven length, against the reference's
    BVHUnion<double, ImplicitFunction<double>, AABB, 4>."""
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built (oracle/_ref)")
    sc = W.csg_scene(11)
    u = BVHUnion(sc["spheres"], [TriMeshSDF(v, f, on_device=True) for v, f in sc["meshes"]], sc["poses"])
    lo = np.minimum(sc["spheres"][:, :3].min(0), sc["poses"][:, 2:5].min(0)) - 0.2
    hi = np.maximum(sc["spheres"][:, :3].max(0), sc["poses"][:, 2:5].max(0)) + 0.2
    rng = np.random.default_rng(12)
    uni = (rng.random((60000, 3)) * (hi - lo) + lo).astype(np.float32)
    near = _near_surface_points(sc, 80, 7, 1e-5)
    p = np.concatenate([uni, near])
    cuts = np.sort(rng.choice(p.shape[0], size=15, replace=False))
    batches = [torch.from_numpy(np.ascontiguousarray(b)).cuda() for b in np.split(p, cuts)]
    d = torch.cat(u.values_batches(batches)).cpu().numpy().astype(np.float64)
    u.check_status()
    ref = oracle.ref().scene(sc["spheres"], sc["meshes"], sc["poses"], _world_boxes(sc)).value(p.astype(np.float64))
    diag = scene_diag(sc["spheres"], sc["meshes"], sc["poses"])
    check(d, ref, diag, "configuration scene")
    inband = np.abs(ref) <= 1e-4 * diag
    clear = inband & (np.abs(ref) > 1e-12)
    assert clear.sum() > 1000
    assert np.all(np.sign(d[clear]) == np.sign(ref[clear]))
