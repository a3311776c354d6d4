"""Parity of the CUDA mesh signed-distance path (through the C ABI) with the reference.

Contract (per query): |d_gpu - d_ref| <= 1e-6 * diag, where diag is the mesh bounding-box
diagonal; the sign equals the reference's wherever |d_ref| > 1e-4 * diag (outside the
near-surface band, where the sign is well conditioned).  The reference values come from the
committed golden fixtures or from the reference library compiled into oracle/_ref."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6   # distance tolerance, x diagonal
BAND = 1e-4      # sign-agreement band, x diagonal


def check_parity(d_gpu, d_ref, diag, what=""):
    d_gpu = np.asarray(d_gpu, np.float64)
    err = np.abs(d_gpu - d_ref)
    assert np.all(np.isfinite(d_gpu)), what
    assert err.max() <= REL_TOL * diag, f"{what}: max err {err.max():.3e} > {REL_TOL * diag:.3e}"
    out = np.abs(d_ref) > BAND * diag
    bad = np.sum(np.sign(d_gpu[out]) != np.sign(d_ref[out]))
    assert bad == 0, f"{what}: {bad} sign mismatches outside the band"


def gpu_sdf(mesh, p, **kw):
    t = torch.from_numpy(np.ascontiguousarray(p, np.float32)).cuda()
    d = mesh.signed_distance(t, **kw)
    torch.cuda.synchronize()
    mesh.check_status()
    return d.cpu().numpy()


@pytest.fixture(scope="module")
def ref():
    return oracle.ref()


@pytest.mark.parametrize("name", ["dodecahedron.npz", "icosphere_l2.npz"])
@pytest.mark.parametrize("build", ["SAH", "Morton"])
def test_golden_meshes(golden, name, build):
    g = golden(name)
    m = TriMeshSDF(g["v"], g["f"], build=build, leaf_size=4)
    fn, vn, en = m.normals()
    assert np.array_equal(fn, g["face_n"]) and np.array_equal(vn, g["vert_n"]) and np.array_equal(en, g["edge_n"])
    # fixture points are float32-representable, so the GPU sees exactly the reference's inputs
    check_parity(gpu_sdf(m, g["p"]), g["ref"], m.diagonal, name)
    # host entry point (e2e path) gives the same numbers
    dh = m.signed_distance(g["p"].astype(np.float32))
    check_parity(dh, g["ref"], m.diagonal, name + " host")


def test_triangle_kats(golden):
    k = golden("triangle_kat.npz")
    for i in range(len(k["expected"])):
        m = TriMeshSDF(k["v"][i], np.array([[0, 1, 2]]), vertex_normals=k["vn"][i][None],
                       edge_normals=k["en"][i][None])
        d = m.value(k["p"][i])
        assert d == pytest.approx(k["expected"][i], abs=1e-6), i


@pytest.mark.parametrize("leaf", [1, 3, 8, 16, 32])
def test_leaf_sizes_and_orders(ref, leaf):
    v, f = W.displaced_icosphere(3, 21)
    p = np.concatenate([W.uniform_points(20000, 22), W.band_points(v, f, 5000, 23)])
    d_ref = ref.mesh(v, f).sdf(p.astype(np.float64))
    m = TriMeshSDF(v, f, leaf_size=leaf)
    check_parity(gpu_sdf(m, p), d_ref, m.diagonal, f"leaf {leaf}")
    check_parity(gpu_sdf(m, p, sort=False), d_ref, m.diagonal, f"leaf {leaf} unsorted")
    for wpb in (1, 2, 8):
        check_parity(gpu_sdf(m, p, warps_per_block=wpb), d_ref, m.diagonal, f"wpb {wpb}")


def test_level5_mesh_uniform_and_band(ref):
    v, f = W.displaced_icosphere(5, 1)  # the CPU-runnable 20,480-triangle configuration
    p = np.concatenate([W.uniform_points(200000, 2), W.band_points(v, f, 50000, 3)])
    d_ref = ref.mesh(v, f, kind=0, build=0, max_leaf_groups=4).sdf(p.astype(np.float64))
    m = TriMeshSDF(v, f)
    d = gpu_sdf(m, p)
    check_parity(d, d_ref, m.diagonal, "L5")
    # closest triangle: its own FP64 distance must equal the reported one within tolerance
    t = torch.from_numpy(p[:2000]).cuda()
    tri = torch.empty(2000, dtype=torch.int32, device="cuda")
    d2, tri = m.signed_distance(t, closest_tri=tri)
    tri = tri.cpu().numpy()
    assert tri.min() >= 0 and tri.max() < f.shape[0]
    P = oracle.port()
    fn, vn, en = m.normals()
    for i in range(0, 2000, 97):
        dt = P.triangle_sd(v[f[tri[i]]], fn[tri[i]], vn[tri[i]], en[tri[i]], p[i].astype(np.float64))
        assert abs(dt - d_ref[i]) <= REL_TOL * m.diagonal


def test_fp64_band_matches_reference_closely(ref):
    v, f = W.displaced_icosphere(4, 5)
    p = W.band_points(v, f, 20000, 6, width=2e-4)  # all inside the default band
    d_ref = ref.mesh(v, f).sdf(p.astype(np.float64))
    m = TriMeshSDF(v, f)
    d = gpu_sdf(m, p)
    # FP64 re-evaluation: error is the float32 rounding of the output only
    assert np.max(np.abs(d - d_ref) / np.maximum(np.abs(d_ref), 1e-30)) <= 1e-6
    assert np.mean(np.sign(d) == np.sign(d_ref)) > 0.999
    d32 = gpu_sdf(m, p, fp64_band=False)
    check_parity(d32, d_ref, m.diagonal, "no band")


@pytest.mark.parametrize("n", [1, 31, 32, 33, 1000])
def test_sizes(ref, n):
    v, f = W.displaced_icosphere(2, 8)
    p = W.uniform_points(n, 9)
    d_ref = ref.mesh(v, f).sdf(p.astype(np.float64))
    m = TriMeshSDF(v, f)
    check_parity(gpu_sdf(m, p), d_ref, m.diagonal, f"n={n}")


def test_tiny_meshes(ref):
    # single triangle (root is a leaf) and a tetrahedron
    tv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    tf = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]])
    p = W.uniform_points(3000, 4, -2, 2)
    m = TriMeshSDF(tv, tf)
    check_parity(gpu_sdf(m, p), ref.mesh(tv, tf).sdf(p.astype(np.float64)), m.diagonal, "tetra")
    assert m.info["num_nodes"] == 0  # 4 triangles fit one leaf


def test_empty_and_errors():
    v, f = W.displaced_icosphere(1, 1)
    m = TriMeshSDF(v, f)
    out = m.signed_distance(torch.empty((0, 3), device="cuda"))
    assert out.numel() == 0
    with pytest.raises(EbgError):
        m.signed_distance(np.array([[np.nan, 0, 0]], np.float32))
    with pytest.raises(EbgError):
        TriMeshSDF(v, np.array([[0, 1, 10 ** 6]]))
    with pytest.raises(EbgError):
        TriMeshSDF(v, f, leaf_size=64)


def test_value_single_point(ref, golden):
    g = golden("dodecahedron.npz")
    m = TriMeshSDF(g["v"], g["f"])
    for i in range(10):
        assert m.value(g["p"][i]) == pytest.approx(g["ref"][i], abs=REL_TOL * m.diagonal)


def test_stats_counters():
    v, f = W.displaced_icosphere(4, 2)
    m = TriMeshSDF(v, f)
    p = torch.from_numpy(W.uniform_points(10000, 3)).cuda()
    d, st = m.stats(p)
    assert st["nodes_visited"] > 10000 and st["triangles_tested"] > st["leaves_visited"] > 0
    assert st["seed_fallbacks"] == 0


def test_level8_properties_full_size():
    """Size-independent properties on the 1,310,720-triangle mesh over 2M grid points: finite,
    1-Lipschitz between grid neighbours, and the sign agrees with the analytic displaced-sphere
    surface for points farther than 1e-3 from it."""
    v, f = W.displaced_icosphere(8, 1)
    m = TriMeshSDF(v, f, build="Morton")
    res = 128
    p = W.grid_points(res, -1.25, 1.25)
    d = gpu_sdf(m, p).reshape(res, res, res)
    assert np.all(np.isfinite(d))
    h = 2.5 / res
    for ax in range(3):
        assert np.max(np.abs(np.diff(d, axis=ax))) <= h * (1 + 1e-5) + 1e-6
    a, w, phi = W.radial_field(1)
    pp = p.astype(np.float64)
    r = np.linalg.norm(pp, axis=1)
    u = pp / np.maximum(r, 1e-12)[:, None]
    rs = 1.0 + (np.sin(u @ w.T + phi) * a).sum(axis=1)
    far = np.abs(r - rs) > 1e-3
    assert np.all(np.sign(d.ravel()[far]) == np.sign(r - rs)[far])


def test_cuda_graph_capture(ref):
    """The query path issues only stream-ordered work (launches, stream-ordered allocations, the
    radix sort), so a caller can capture it once and replay it."""
    v, f = W.displaced_icosphere(4, 31)
    m = TriMeshSDF(v, f)
    p = W.uniform_points(50000, 32)
    d_ref = ref.mesh(v, f).sdf(p.astype(np.float64))
    pd = torch.from_numpy(p).cuda()
    out = torch.empty(p.shape[0], device="cuda")
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(2):
            m.signed_distance(pd, out=out, stream=s)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        m.signed_distance(pd, out=out, stream=s)
    out.zero_()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    check_parity(out.cpu().numpy(), d_ref, m.diagonal, "graph replay")


def test_chunked_host_call_matches_device_path():
    """Host calls of more than 4M points run in overlapping chunks on two streams; the results are
    those of the one-piece device call, including the closest triangles and a per-point hint."""
    v, f = W.displaced_icosphere(4, 41)
    m = TriMeshSDF(v, f)
    p = W.uniform_points(5_000_000, 42)
    pd = torch.from_numpy(p).cuda()
    tri_d = torch.empty(p.shape[0], dtype=torch.int32, device="cuda")
    d_dev, _ = m.signed_distance(pd, closest_tri=tri_d)
    torch.cuda.synchronize()
    d_host, tri_h = m.signed_distance(p, closest_tri=np.empty(p.shape[0], np.int32))
    assert np.array_equal(d_host, d_dev.cpu().numpy())
    assert np.array_equal(tri_h, tri_d.cpu().numpy())
    hint = (d_dev.abs() * 1.01 + 1e-3).contiguous()
    d_hint = m.signed_distance(p, radius_hint=hint)
    assert np.array_equal(d_hint, d_host)


def test_ramped_host_call_matches_device_path():
    """Host calls of at least 64M points use ramped chunks (1, 2, 4 units, pieces of about 8, then
    4, 2, 1; a unit is 1/64 of the call) with a last chunk that is not a multiple of 32 points: the
    results are still those of the one-piece device call."""
    v, f = W.displaced_icosphere(2, 43)
    m = TriMeshSDF(v, f)
    n = (1 << 26) + 45
    p = np.random.default_rng(44).uniform(-1.5, 1.5, size=(n, 3)).astype(np.float32)
    pd = torch.from_numpy(p).cuda()
    tri_d = torch.empty(n, dtype=torch.int32, device="cuda")
    d_dev, _ = m.signed_distance(pd, closest_tri=tri_d)
    torch.cuda.synchronize()
    d_host, tri_h = m.signed_distance(p, closest_tri=np.empty(n, np.int32))
    assert np.array_equal(d_host, d_dev.cpu().numpy())
    assert np.array_equal(tri_h, tri_d.cpu().numpy())


@pytest.mark.parametrize("on_device", [True, False])
def test_top_nodes_in_shared_memory_change_nothing(ref, on_device):
    """Plain queries that read the tree's top nodes from each block's shared-memory copy
    (ebg_query_opts.top_nodes) give the results and closest triangles of the default path, for
    the level-ordered device build and the host build, up to more nodes than the tree has."""
    v, f = W.displaced_icosphere(6, 51)
    m = TriMeshSDF(v, f, build="Morton", on_device=on_device)
    p = np.concatenate([W.uniform_points(300000, 52), W.band_points(v, f, 50000, 53)])
    pd = torch.from_numpy(p).cuda()
    tri0 = torch.empty(p.shape[0], dtype=torch.int32, device="cuda")
    d0, _ = m.signed_distance(pd, closest_tri=tri0)
    for top in (1, 21, 85, 512, 100000):
        tri = torch.empty_like(tri0)
        d, _ = m.signed_distance(pd, closest_tri=tri, top_nodes=top)
        torch.cuda.synchronize()
        m.check_status()
        assert torch.equal(d, d0), top
        assert torch.equal(tri, tri0), top
    d_ref = ref.mesh(v, f, kind=0, build=1, max_leaf_groups=4).sdf(p[:20000].astype(np.float64))
    check_parity(d0[:20000].cpu().numpy(), d_ref, m.diagonal, "L6 top nodes")
