"""The allocation-free mesh query, ebg_mesh_signed_distance_noalloc, through the C ABI.

Callers such as AMR codes that reserve the GPU's memory for their own arena at start-up cannot let a
library allocate device memory inside their embedded-boundary loop; this entry point takes its
workspace from a fixed array compiled into the library.  The tests check, on two calls in a row (the
array keeps the previous call's contents), that its distances match the allocating entry point's and
the reference's within the parity tolerance, also at the size limit with a seed model attached; that
it allocates nothing from the device's memory pool (the pool's high-water marks do not move, while
they do for the allocating entry point); that a call with no points prepares the array, also in a
fresh process with lazy module loading; and that it rejects a batch above its size limit.  The file
is collected last, and passes alone in a fresh process as well as after the others."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle
from conftest import ROOT
from ebgeometry_b200 import SeedModel, TriMeshSDF, _capi
from ebgeometry_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_POINTS = 1 << 19


def _noalloc(mesh, pts, out, opts=None, n=None):
    o = opts if opts is not None else _capi.QueryOpts()
    count = pts.shape[0] if n is None else n
    return _capi.lib.ebg_mesh_signed_distance_noalloc(
        mesh.handle, C.c_void_p(pts.data_ptr()), count, C.c_void_p(out.data_ptr()), None, C.byref(o),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))


class _PoolWatermarks:
    """High-water marks of the current device's default memory pool (the pool the allocating entry
    point takes its workspace from): reset before a call, read after it."""

    def __init__(self):
        try:
            from cuda.bindings import driver, runtime
        except ImportError:
            pytest.skip("cuda-python is not installed: the memory pool's high-water marks cannot be read")
        self.rt, self.drv = runtime, driver
        err, dev = runtime.cudaGetDevice()
        err, self.pool = runtime.cudaDeviceGetDefaultMemPool(dev)
        if err != runtime.cudaError_t.cudaSuccess:
            pytest.skip("no default memory pool on this device")
        self.attrs = (runtime.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                      runtime.cudaMemPoolAttr.cudaMemPoolAttrReservedMemHigh)

    def reset(self):
        torch.cuda.synchronize()
        for a in self.attrs:
            (err,) = self.rt.cudaMemPoolSetAttribute(self.pool, a, self.drv.cuuint64_t(0))
            assert err == self.rt.cudaError_t.cudaSuccess, err
        return self.read()

    def read(self):
        torch.cuda.synchronize()
        vals = []
        for a in self.attrs:
            err, v = self.rt.cudaMemPoolGetAttribute(self.pool, a)
            assert err == self.rt.cudaError_t.cudaSuccess, err
            vals.append(int(v))
        return tuple(vals)


def _parity(d, ref, diag):
    """Largest |d - ref| and the sign mismatches outside the near-surface band."""
    d = np.asarray(d, np.float64)
    outside = np.abs(ref) > 1e-4 * diag
    return float(np.abs(d - ref).max()), int(np.sum(np.sign(d[outside]) != np.sign(ref[outside])))


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
        assert _noalloc(mesh, pts, out) == 0, _capi.lib.ebg_last_error().decode()
        torch.cuda.synchronize()
        mesh.check_status()
        assert torch.isfinite(out).all()
        err = (out - ref).abs().max().item()
        assert err <= tol, (i, err, tol)


def test_noalloc_allocates_nothing_and_the_allocating_path_does():
    v, f = W.displaced_icosphere(4, 5)
    mesh = TriMeshSDF(v, f)
    pts = torch.from_numpy(W.uniform_points(200000, 21)).cuda()
    out = torch.empty(pts.shape[0], device="cuda")
    assert _noalloc(mesh, pts, out) == 0  # the first call on the device sets the array up
    pool = _PoolWatermarks()
    before = pool.reset()
    assert _noalloc(mesh, pts, out) == 0, _capi.lib.ebg_last_error().decode()
    assert pool.read() == before, "the allocation-free entry point took memory from the pool"
    # control: the same check catches the allocating entry point's workspace
    before = pool.reset()
    mesh.signed_distance(pts, out=out)
    after = pool.read()
    assert after[0] > before[0], (before, after)


def test_noalloc_at_the_size_limit_with_a_seed_against_the_reference():
    if not oracle.ref_available():
        pytest.skip("reference oracle library not built (oracle/_ref)")
    v, f = W.displaced_icosphere(5, 8)
    mesh = TriMeshSDF(v, f)
    seed = SeedModel.train(mesh, num_samples=1 << 18, steps=300, batch=1 << 14, rng_seed=3,
                           lo=[-1.25] * 3, hi=[1.25] * 3)
    mesh.attach_seed(seed, cells_per_axis=32)
    p = np.concatenate([W.uniform_points(MAX_POINTS - 100000, 31, -1.25, 1.25), W.band_points(v, f, 100000, 32)])
    assert p.shape[0] == MAX_POINTS
    pts = torch.from_numpy(p).cuda()
    opts = _capi.QueryOpts()
    opts.seed = seed.handle
    ref_mesh = oracle.ref().mesh(v, f, kind=0, build=0, max_leaf_groups=4)  # TriMeshSDF<double,short,4,4>, SAH
    d_ref = ref_mesh.sdf(p.astype(np.float64))
    plain = mesh.signed_distance(pts).cpu().numpy()
    for call in range(2):
        out = torch.full((MAX_POINTS,), float("nan"), device="cuda")
        assert _noalloc(mesh, pts, out, opts) == 0, _capi.lib.ebg_last_error().decode()
        torch.cuda.synchronize()
        mesh.check_status()
        d = out.cpu().numpy()
        err, signs = _parity(d, d_ref, mesh.diagonal)
        assert err <= 1e-6 * mesh.diagonal and signs == 0, (call, err, signs)
        assert np.array_equal(d, plain), call  # seeded results are the plain traversal's


def test_noalloc_empty_call_sets_up_in_a_fresh_lazy_process():
    code = r"""
import sys, numpy as np, torch, ctypes as C
sys.path.insert(0, sys.argv[1])
from ebgeometry_b200 import TriMeshSDF, _capi
from ebgeometry_b200 import workloads as W
v, f = W.displaced_icosphere(3, 2)
mesh = TriMeshSDF(v, f)
s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
o = _capi.QueryOpts()
assert _capi.lib.ebg_mesh_signed_distance_noalloc(mesh.handle, None, 0, None, None, C.byref(o), s) == 0
pts = torch.from_numpy(W.uniform_points(50000, 4)).cuda()
out = torch.empty(50000, device="cuda")
assert _capi.lib.ebg_mesh_signed_distance_noalloc(mesh.handle, C.c_void_p(pts.data_ptr()), 50000,
                                                  C.c_void_p(out.data_ptr()), None, C.byref(o), s) == 0
ref = mesh.signed_distance(pts)
torch.cuda.synchronize()
assert (out - ref).abs().max().item() <= 1e-6 * mesh.diagonal
print("ok")
"""
    env = dict(os.environ, CUDA_MODULE_LOADING="LAZY")
    r = subprocess.run([sys.executable, "-c", code, ROOT], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr


def test_noalloc_rejects_too_many_points():
    v, f = W.displaced_icosphere(2, 3)
    mesh = TriMeshSDF(v, f)
    pts = torch.zeros((MAX_POINTS + 1, 3), device="cuda")
    out = torch.empty(MAX_POINTS + 1, device="cuda")
    rc = _noalloc(mesh, pts, out)
    assert rc == 6 and b"at most" in _capi.lib.ebg_last_error()  # EBG_ERR_TOO_LARGE
