"""Queries through the 8-wide copy of the tree (ebg_mesh_widen, ebg_query_opts.node_width = 8).

The copy keeps the 4-wide tree's leaves and child boxes, and both traversals break distance ties
by the lower leaf position, so every distance and closest triangle must equal the 4-wide
traversal's bit for bit; against the reference the usual parity contract holds (|d - d_ref| <=
1e-6 x diagonal, signs equal outside the 1e-4 x diagonal band).  Also: both build methods on the
host and on the device, leaf sizes, radius hints and FP64 calls through the copy; a mesh whose root
is a leaf; node_width 8 without a copy is rejected; a refit drops the copy; the autotuner's node
width axis keeps the answers."""
import numpy as np
import pytest
import torch

import oracle
from ebgeometry_b200 import EbgError, TriMeshSDF
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6
BAND = 1e-4


def _points(v, f, n_uniform, n_band, seed):
    return torch.from_numpy(np.concatenate([W.uniform_points(n_uniform, seed, -1.25, 1.25),
                                            W.band_points(v, f, n_band, seed + 1)])).cuda()


def _both(mesh, p, **kw):
    t4 = torch.empty(p.shape[0], dtype=torch.int32, device="cuda")
    t8 = torch.empty_like(t4)
    d4, t4 = mesh.signed_distance(p, closest_tri=t4, node_width=4, **kw)
    d8, t8 = mesh.signed_distance(p, closest_tri=t8, node_width=8, **kw)
    torch.cuda.synchronize()
    mesh.check_status()
    return d4, t4, d8, t8


@pytest.mark.parametrize("level,build,on_device,leaf", [(5, "SAH", False, 8), (5, "Morton", True, 8),
                                                        (6, "SAH", True, 4), (7, "Morton", True, 8),
                                                        (4, "Morton", False, 1), (4, "SAH", False, 16)])
def test_eight_wide_equals_four_wide(level, build, on_device, leaf):
    v, f = W.displaced_icosphere(level, 3)
    mesh = TriMeshSDF(v, f, build=build, leaf_size=leaf, on_device=on_device)
    info = mesh.widen()
    assert 0 < info["num_nodes8"] < mesh.info["num_nodes"]
    assert info["depth8"] <= mesh.info["depth"] + 1
    p = _points(v, f, 200000, 50000, 7)
    d4, t4, d8, t8 = _both(mesh, p)
    assert torch.equal(d4, d8) and torch.equal(t4, t8)
    # unsorted points, and other launch shapes, through the copy
    assert torch.equal(mesh.signed_distance(p, node_width=8, sort=False), d4)
    for occ, wpb in ((2, 4), (4, 8), (1, 1)):
        assert torch.equal(mesh.signed_distance(p, node_width=8, occupancy=occ, warps_per_block=wpb), d4)
    # the copy opens fewer nodes per packet
    _, s4 = mesh.stats(p, node_width=4)
    _, s8 = mesh.stats(p, node_width=8)
    print(f"L{level} {build} leaf {leaf}: nodes {info['num_nodes8']} of {mesh.info['num_nodes']}, depth "
          f"{info['depth8']} of {mesh.info['depth']}; packet nodes {s8['packet_nodes'] / s8['packets']:.1f} vs "
          f"{s4['packet_nodes'] / s4['packets']:.1f}, pops {s8['packet_pops'] / s8['packets']:.1f} vs "
          f"{s4['packet_pops'] / s4['packets']:.1f}")
    assert s8["packet_nodes"] < s4["packet_nodes"]


def test_eight_wide_against_the_reference():
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built (oracle/_ref)")
    v, f = W.displaced_icosphere(5, 1)
    p = np.concatenate([W.uniform_points(100000, 2), W.band_points(v, f, 30000, 3)])
    d_ref = oracle.ref().mesh(v, f, kind=0, build=0, max_leaf_groups=4).sdf(p.astype(np.float64))
    mesh = TriMeshSDF(v, f)
    mesh.widen()
    d = mesh.signed_distance(torch.from_numpy(p).cuda(), node_width=8).cpu().numpy().astype(np.float64)
    mesh.check_status()
    assert np.abs(d - d_ref).max() <= REL_TOL * mesh.diagonal
    out = np.abs(d_ref) > BAND * mesh.diagonal
    assert int(np.sum(np.sign(d[out]) != np.sign(d_ref[out]))) == 0


def test_eight_wide_hints_and_fp64_calls():
    v, f = W.displaced_icosphere(5, 4)
    mesh = TriMeshSDF(v, f, build="Morton", on_device=True)
    mesh.widen()
    p = _points(v, f, 100000, 30000, 11)
    d4 = mesh.signed_distance(p, node_width=4)
    # radius hints: exact |d| (tight) and a too-small one (second traversal from the root)
    for scale in (1.0001, 0.5):
        hint = (d4.abs() * scale).contiguous()
        assert torch.equal(mesh.signed_distance(p, radius_hint=hint, node_width=8), d4)
    p64 = p.double()
    assert torch.equal(mesh.signed_distance(p64, node_width=8), mesh.signed_distance(p64, node_width=4))
    torch.cuda.synchronize()
    mesh.check_status()


def test_root_leaf_mesh_and_errors():
    # a tetrahedron in one leaf: nothing to widen, width 8 answers as width 4
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float64)
    f = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.int32)
    tet = TriMeshSDF(v, f, leaf_size=4)
    p = torch.from_numpy(W.uniform_points(5000, 3, -1.0, 2.0)).cuda()
    with pytest.raises(EbgError) as e:
        tet.signed_distance(p, node_width=8)  # no copy yet
    assert e.value.status == 1
    assert tet.widen()["num_nodes8"] == 0
    assert torch.equal(tet.signed_distance(p, node_width=8), tet.signed_distance(p, node_width=4))
    with pytest.raises(EbgError) as e:
        tet.signed_distance(p, node_width=6)
    assert e.value.status == 1


def test_refit_drops_the_copy():
    v, f = W.displaced_icosphere(4, 6)
    mesh = TriMeshSDF(v, f)
    mesh.widen()
    p = _points(v, f, 50000, 10000, 21)
    mesh.refit(v * 1.1)
    with pytest.raises(EbgError):
        mesh.signed_distance(p, node_width=8)
    mesh.widen()
    d4, t4, d8, t8 = _both(mesh, p)
    assert torch.equal(d4, d8) and torch.equal(t4, t8)
    d_moved = TriMeshSDF(v * 1.1, f).signed_distance(p)
    assert (d8 - d_moved).abs().max().item() <= REL_TOL * mesh.diagonal


def test_autotune_node_width_axis_keeps_results():
    v, f = W.displaced_icosphere(6, 8)
    mesh = TriMeshSDF(v, f, build="Morton", on_device=True)
    p = _points(v, f, 200000, 50000, 31)
    d0 = mesh.signed_distance(p, node_width=4).clone()
    assert mesh.autotune(p)["node_width"] == 4  # no copy: width 4 only
    mesh.widen()
    r = mesh.autotune(p)
    print("autotune with the 8-wide copy:", r)
    assert r["node_width"] in (4, 8) and r["ms"] > 0
    assert torch.equal(mesh.signed_distance(p), d0)  # the tuned width
    torch.cuda.synchronize()
    mesh.check_status()
