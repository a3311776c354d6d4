"""The autotuner picks a launch shape and a build from measured candidates, the mesh uses it, the
results do not change, and the choice is cached."""
import json

import numpy as np
import pytest
import torch

from ebgeometry_b200 import TriMeshSDF
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
    d1 = m.signed_distance(p)
    torch.cuda.synchronize()
    assert torch.equal(d0, d1)


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
