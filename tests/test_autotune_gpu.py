"""The autotuner picks a launch shape and a build from measured candidates, the mesh uses it, the
results do not change, and the choice is cached."""
import json

import numpy as np
import pytest
import torch

from ebgeometry_b200 import BVHUnion, SeedModel, TriMeshSDF
from ebgeometry_b200 import autotune
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_launch_shape_autotune_keeps_results():
    v, f = W.displaced_icosphere(4, 8)
    m = TriMeshSDF(v, f)
    p = torch.from_numpy(W.uniform_points(100000, 9)).cuda()
    d0 = m.signed_distance(p).clone()
    r = m.autotune(p)
    assert r["occupancy"] in (1, 2, 4) and r["warps_per_block"] in (2, 4, 8) and r["ms"] > 0
    assert r["queue_chunk"] in (1, 2, 4)
    d1 = m.signed_distance(p)
    torch.cuda.synchronize()
    assert torch.equal(d0, d1)
    for chunk in (1, 3, 8):  # any queue chunk gives the same answers
        assert torch.equal(m.signed_distance(p, queue_chunk=chunk), d0)


def test_seeded_autotune_keeps_results():
    v, f = W.displaced_icosphere(4, 8)
    m = TriMeshSDF(v, f)
    seed = SeedModel.train(m, num_samples=1 << 18, steps=200, batch=1 << 14, rng_seed=5, lo=[-1.25] * 3, hi=[1.25] * 3)
    p = torch.from_numpy(W.grid_points(48, -1.25, 1.25)).cuda()
    d0 = m.signed_distance(p)
    r = m.autotune(p, seed=seed)
    assert r["queue_chunk"] in (1, 2, 4) and r["ms"] > 0
    assert torch.equal(m.signed_distance(p, seed=seed), d0)


def test_scene_autotune_keeps_results():
    sc = W.csg_scene(5, n_spheres=200, n_meshes=6, levels=(1, 3), mesh_radius=(0.05, 0.2))
    u = BVHUnion(sc["spheres"], [TriMeshSDF(v, f) for v, f in sc["meshes"]], sc["poses"])
    p = torch.from_numpy(W.uniform_points(100000, 3, -1.2, 1.2)).cuda()
    d0 = u.values(p).clone()
    r = u.autotune(p)
    assert r["queue_chunk"] in (1, 2, 4, 8) and r["ms"] > 0
    assert torch.equal(u.values(p), d0)


def test_build_autotune_and_cache(tmp_path):
    v, f = W.displaced_icosphere(3, 10)
    sample = W.uniform_points(20000, 11)
    cache = str(tmp_path / "tune.json")
    best = autotune.tune_mesh(v, f, sample, builds=("SAH", "Morton"), leaf_sizes=(4, 8), cache_path=cache)
    assert best["build"] in ("SAH", "Morton") and best["leaf_size"] in (4, 8)
    assert len(best["candidates"]) == 4
    assert best["ms"] == min(c["ms"] for c in best["candidates"])
    with open(cache) as fh:
        assert autotune.mesh_key(v, f, len(sample)) in json.load(fh)
    again = autotune.tune_mesh(v, f, sample, cache_path=cache)  # served from the cache
    assert again == best
    mesh, _ = autotune.build_tuned(v, f, sample, cache_path=cache)
    assert mesh.info["leaf_size"] == best["leaf_size"]
