"""The allocation-free mesh query, ebg_mesh_signed_distance_noalloc, through the C ABI.

Callers such as AMR codes that reserve the GPU's memory for their own arena cannot let a library
allocate device memory; this entry point takes its workspace from a fixed array compiled into the
library.  The test checks, on two calls in a row (the array keeps the previous call's contents), that
its distances match the allocating entry point's within the parity tolerance, that it allocates
nothing from the device's memory pool, and that it rejects a batch above its size limit.  It lives in
a file of its own collected last, and passes alone in a fresh process as well as after the others."""
import ctypes as C

import numpy as np
import pytest
import torch

from ebgeometry_b200 import TriMeshSDF, _capi
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_POINTS = 1 << 19


def _noalloc(mesh, pts, out, opts=None):
    o = opts if opts is not None else _capi.QueryOpts()
    return _capi.lib.ebg_mesh_signed_distance_noalloc(
        mesh.handle, C.c_void_p(pts.data_ptr()), pts.shape[0], C.c_void_p(out.data_ptr()), None, C.byref(o),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))


def _pool_used_bytes():
    """Bytes in use in the current device's default memory pool (None without cuda-python)."""
    try:
        from cuda.bindings import runtime as cudart
    except ImportError:
        try:
            from cuda import cudart
        except ImportError:
            return None
    err, dev = cudart.cudaGetDevice()
    err, pool = cudart.cudaDeviceGetDefaultMemPool(dev)
    if err != cudart.cudaError_t.cudaSuccess:
        return None
    err, used = cudart.cudaMemPoolGetAttribute(pool, cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    return int(used) if err == cudart.cudaError_t.cudaSuccess else None


def test_noalloc_matches_allocating_entry_point_twice():
    v, f = W.displaced_icosphere(5, 3)
    mesh = TriMeshSDF(v, f)
    tol = 1e-6 * mesh.diagonal
    batches = [np.concatenate([W.uniform_points(300000, 11), W.band_points(v, f, 40000, 12)]),
               np.concatenate([W.grid_points(64, -1.25, 1.25), W.band_points(v, f, 20000, 13)])]
    for i, b in enumerate(batches):  # two calls in a row: the second sees the first call's leftovers
        pts = torch.from_numpy(b).cuda()
        ref = mesh.signed_distance(pts)
        torch.cuda.synchronize()
        out = torch.full_like(ref, float("nan"))
        before = _pool_used_bytes()
        assert _noalloc(mesh, pts, out) == 0, _capi.lib.ebg_last_error().decode()
        torch.cuda.synchronize()
        after = _pool_used_bytes()
        mesh.check_status()
        assert torch.isfinite(out).all()
        err = (out - ref).abs().max().item()
        assert err <= tol, (i, err, tol)
        if before is not None:
            assert after == before, (before, after)


def test_noalloc_rejects_too_many_points():
    v, f = W.displaced_icosphere(2, 3)
    mesh = TriMeshSDF(v, f)
    pts = torch.zeros((MAX_POINTS + 1, 3), device="cuda")
    out = torch.empty(MAX_POINTS + 1, device="cuda")
    rc = _noalloc(mesh, pts, out)
    assert rc == 6 and b"at most" in _capi.lib.ebg_last_error()  # EBG_ERR_TOO_LARGE
