"""Autotuner for the mesh query path (no reference counterpart).

Two levels: the BVH's build method and leaf size (fixed when a mesh is built, so each candidate is
a rebuild), and, inside the library (``ebg_mesh_autotune``), the traversal's launch shape (register
budget x warps per block), the work-queue chunk and the node width (the 4-wide tree or its 8-wide
copy, ``ebg_mesh_widen``).  The winner is cached in a JSON file keyed by a hash of the mesh
and the sample size, so later runs build the tuned mesh directly.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np


def mesh_key(vertices, triangles, n_sample: int) -> str:
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(vertices, np.float64).tobytes())
    h.update(np.ascontiguousarray(triangles, np.int32).tobytes())
    h.update(str(n_sample).encode())
    return h.hexdigest()


def tune_mesh(vertices, triangles, sample_points, builds=("SAH", "Morton"), leaf_sizes=(4, 8, 12, 16),
              cache_path=None, device=0, widths=(4, 8)):
    """Returns {"build", "leaf_size", "occupancy", "warps_per_block", "queue_chunk", "node_width", "ms",
    "candidates"}: the fastest plain traversal of the sample (float32 (n,3) numpy array) over the
    candidates.  ``widths`` containing 8 lets each candidate also time its tree's 8-wide copy."""
    import torch

    from . import EbgError, TriMeshSDF
    key = mesh_key(vertices, triangles, len(sample_points))
    cache = {}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as fh:
            cache = json.load(fh)
        if key in cache:
            return cache[key]
    pts = torch.from_numpy(np.ascontiguousarray(sample_points, np.float32)).to(f"cuda:{device}")
    cands = []
    for b in builds:
        for leaf in leaf_sizes:
            mesh = TriMeshSDF(vertices, triangles, build=b, leaf_size=leaf, device=device)
            if 8 in widths:
                try:
                    mesh.widen()
                except EbgError:
                    pass  # a tree too deep for the 8-wide stack keeps width 4
            r = mesh.autotune(pts)
            cands.append({"build": b, "leaf_size": leaf, **r})
            del mesh
    best = dict(min(cands, key=lambda c: c["ms"]))
    best["candidates"] = cands
    if cache_path:
        cache[key] = best
        tmp = cache_path + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(cache, fh, indent=1)
        os.replace(tmp, cache_path)
    return best


def build_tuned(vertices, triangles, sample_points, cache_path=None, device=0, **kw):
    """A TriMeshSDF built and launched with the tuned configuration."""
    import torch

    from . import TriMeshSDF
    best = tune_mesh(vertices, triangles, sample_points, cache_path=cache_path, device=device, **kw)
    mesh = TriMeshSDF(vertices, triangles, build=best["build"], leaf_size=best["leaf_size"], device=device)
    if best.get("node_width") == 8:
        mesh.widen()
    mesh.autotune(torch.from_numpy(np.ascontiguousarray(sample_points, np.float32)).to(f"cuda:{device}"))
    return mesh, best
