"""ebgeometry_b200 -- B200-native (sm_100a) mesh signed distance, nearest neighbours and CSG union.

Python mirror of the reference's (rmrsk/EBGeometry) C++ query objects on top of the C ABI in
``include/ebgeometry_b200.h``.  Class and method names follow the reference:

* :class:`TriMeshSDF` -- ``TriMeshSDF(mesh, build, maxLeafGroups)`` (MeshDistanceFunctions.hpp:
  309-489) with ``value(point)`` / ``signedDistance(point)`` for one point (ImplicitFunction.hpp:
  51-60) and a batched ``signed_distance(points)`` over CUDA tensors or numpy arrays.
* :class:`PointCloudBVH` -- ``PointCloudBVH(positions, meta)`` (PointCloudBVH.hpp:56-350) with
  ``closestPoint`` / ``closestPoints`` for one point and a batched ``knn(queries, k)``.
* :class:`BVHUnion` -- ``BVHUnion(prims, bvs)`` (CSG.hpp:99-101) over spheres and
  ``Translate(Rotate(TriMeshSDF))`` instances, with ``value(point)`` and batched ``values(points)``.

There is no CPU fallback: every query runs in the CUDA kernels of ``libebgb200.so``, and importing
this package fails if that library is missing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import EbgError, check, lib

__all__ = ["sample_points", "read_soup", "read_polygon_soup", "TriMeshSDF", "MeshSDF", "FlatMeshSDF", "PolygonMeshSDF",
           "PolygonFlatMeshSDF", "polygon_normals", "PointCloudBVH", "PointCloudHashGrid",
           "BVHUnion", "SeedModel", "EbgError", "BUILD_SAH", "BUILD_MORTON", "version", "device_count"]

BUILD_SAH = 0
BUILD_MORTON = 1


def version() -> str:
    return lib.ebg_version().decode()


def device_count() -> int:
    return int(lib.ebg_device_count())


def sample_points(n: int, seed: int) -> np.ndarray:
    """Random::samplePoints<double>(n, seed) (RandomImplem.hpp:27-44): the reference's seeded
    points uniform in [0,1)^3, float64 (n,3)."""
    out = np.empty((int(n), 3), np.float64)
    check(lib.ebg_sample_points(int(n), C.c_uint64(int(seed)), _ptr(out)))
    return out


def read_soup(path):
    """(vertices (V,3) float64, triangles (T,3) int32) of a mesh file (.stl, .obj, .ply, .vtk) read
    and merged the way the reference's parser does (host only, no device needed)."""
    h = C.c_void_p()
    check(lib.ebg_soup_read(str(path).encode(), C.byref(h)))
    try:
        nv, nt = C.c_int64(), C.c_int64()
        check(lib.ebg_soup_sizes(h, C.byref(nv), C.byref(nt)))
        v = np.empty((nv.value, 3), np.float64)
        f = np.empty((nt.value, 3), np.int32)
        check(lib.ebg_soup_copy(h, _ptr(v), _ptr(f)))
    finally:
        lib.ebg_soup_destroy(h)
    return v, f


def read_polygon_soup(path):
    """(vertices (V,3) float64, face offsets (F+1,) int64, face vertex indices int32) of a mesh file
    of any faces, read and merged the way the reference's parser does (host only)."""
    h = C.c_void_p()
    check(lib.ebg_soup_read(str(path).encode(), C.byref(h)))
    try:
        nv, nf, nc = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib.ebg_soup_sizes(h, C.byref(nv), C.byref(nf)))
        check(lib.ebg_soup_num_corners(h, C.byref(nc)))
        v = np.empty((nv.value, 3), np.float64)
        off = np.empty(nf.value + 1, np.int64)
        idx = np.empty(nc.value, np.int32)
        check(lib.ebg_soup_copy_polygons(h, _ptr(v), _ptr(off), _ptr(idx)))
    finally:
        lib.ebg_soup_destroy(h)
    return v, off, idx


def _stream_ptr(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class TriMeshSDF:
    """Signed distance to a watertight triangle mesh (the reference's TriMeshSDF).

    ``vertices``: (V,3) float64; ``triangles``: (T,3) int32 corner indices, counter-clockwise seen
    from outside.  Pseudonormals are computed the way the reference's DCEL computes them unless
    ``vertex_normals`` (per corner, (T,3,3)) and ``edge_normals`` ((T,3,3), edge i from corner i to
    i+1) are given.  ``build``: "SAH" or "Morton"; ``leaf_size``: max triangles per leaf;
    ``on_device``: build the tree (either method; the host build's tree), pseudonormals, records and
    boxes on the GPU.
    """

    def __init__(self, vertices, triangles, build="SAH", leaf_size=8, device=-1,
                 vertex_normals=None, edge_normals=None, on_device=False):
        v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        f = np.ascontiguousarray(triangles, dtype=np.int32).reshape(-1, 3)
        b = {"SAH": BUILD_SAH, "MORTON": BUILD_MORTON}[str(build).upper()] if isinstance(build, str) else int(build)
        opts = _capi.BuildOpts(b, int(leaf_size), int(device), 1 if on_device else 0)
        h = C.c_void_p()
        if vertex_normals is not None or edge_normals is not None:
            vn = np.ascontiguousarray(vertex_normals, dtype=np.float64).reshape(-1, 9)
            en = np.ascontiguousarray(edge_normals, dtype=np.float64).reshape(-1, 9)
            if vn.shape[0] != f.shape[0] or en.shape[0] != f.shape[0]:
                raise ValueError("one row of 9 normal components per triangle expected")
            check(lib.ebg_mesh_create_with_normals(_ptr(v), v.shape[0], _ptr(f), f.shape[0], _ptr(vn),
                                                   _ptr(en), C.byref(opts), C.byref(h)))
        else:
            check(lib.ebg_mesh_create(_ptr(v), v.shape[0], _ptr(f), f.shape[0], C.byref(opts),
                                      C.byref(h)))
        self._h = h
        self.num_triangles = f.shape[0]
        self._refresh_info()

    @classmethod
    def from_file(cls, path, **kw):
        """Parser::readIntoTriangleBVH: the mesh of a .stl / .obj / .ply / .vtk file."""
        v, f = read_soup(path)
        return cls(v, f, **kw)

    def _refresh_info(self):
        inf = _capi.MeshInfo()
        check(lib.ebg_mesh_get_info(self._h, C.byref(inf)))
        self.info = {k: (list(getattr(inf, k)) if k in ("lo", "hi") else getattr(inf, k))
                     for k, _ in _capi.MeshInfo._fields_}

    def refit(self, vertices, stream=None):
        """PackedBVH::refit for moved vertices: ``vertices`` (V,3) float64 -- numpy, or a CUDA
        tensor -- are the new positions of the same vertices.  The tree keeps its topology; normals,
        records and boxes are recomputed on the device, so later queries are exact for the moved
        mesh.  Synchronous."""
        if isinstance(vertices, np.ndarray) or not hasattr(vertices, "is_cuda"):
            v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
            check(lib.ebg_mesh_refit(self._h, _ptr(v), v.shape[0], _stream_ptr(stream)))
        else:
            import torch
            if not (vertices.is_cuda and vertices.dtype == torch.float64 and vertices.is_contiguous()):
                raise ValueError("vertices must be a contiguous float64 CUDA tensor of shape (V,3)")
            check(lib.ebg_mesh_refit_device(self._h, C.c_void_p(vertices.data_ptr()), vertices.numel() // 3,
                                            _stream_ptr(stream)))
        self._refresh_info()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.ebg_mesh_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def diagonal(self) -> float:
        return float(self.info["diagonal"])

    def normals(self):
        """(face (T,3), corner vertex (T,3,3), edge (T,3,3)) pseudonormals as float64."""
        t = self.num_triangles
        fn, vn, en = np.empty((t, 3)), np.empty((t, 3, 3)), np.empty((t, 3, 3))
        check(lib.ebg_mesh_get_normals(self._h, _ptr(fn), _ptr(vn), _ptr(en)))
        return fn, vn, en

    @staticmethod
    def _opts(band, sort, fp64_band, warps_per_block, timings=None, seed=None, radius_hint=None, occupancy=None,
              queue_chunk=None, top_nodes=None, node_width=None):
        return _capi.QueryOpts(float(band or 0.0), 0 if sort else 1, 0 if fp64_band else 1,
                               seed.handle if seed is not None else None,
                               int(warps_per_block or 0), int(occupancy or 0),
                               C.pointer(timings) if timings is not None else None,
                               radius_hint.data_ptr() if radius_hint is not None else None, int(queue_chunk or 0),
                               int(top_nodes or 0), int(node_width or 0))

    # --- ImplicitFunction<T>::value / SignedDistanceFunction<T>::signedDistance -----------------
    def value(self, point) -> float:
        out = C.c_double()
        check(lib.ebg_mesh_value(self._h, float(point[0]), float(point[1]), float(point[2]),
                                 C.byref(out)))
        return out.value

    signedDistance = value
    __call__ = value

    # --- batched ----------------------------------------------------------------------------------
    def signed_distance(self, points, out=None, closest_tri=None, band=None, sort=True,
                        fp64_band=True, warps_per_block=None, stream=None, timings=None, seed=None,
                        radius_hint=None, occupancy=None, queue_chunk=None, top_nodes=None, node_width=None):
        """Signed distances of (n,3) float32 points.  CUDA tensors stay on the device (asynchronous
        on ``stream``, default the current torch stream); numpy arrays go through the host entry
        point (synchronous).  Float64 points (numpy or CUDA) take the FP64 entry points: every
        query is re-evaluated in FP64 and the distances come back as float64.  ``timings``: an ``_capi.PhaseTimings`` to fill with per-phase device
        times (the call then synchronises).  ``seed``: a trained :class:`SeedModel` whose predicted
        radius seeds the traversal's pruning bound (results stay exact).  ``radius_hint``: a CUDA
        float32 tensor of per-point upper bounds on |d| that seed the bound the same way.
        ``top_nodes``: plain queries read the tree's first ``top_nodes`` nodes from a copy in each
        block's shared memory (ebg_query_opts.top_nodes; same results).  ``node_width``: 8 traverses
        the 8-wide copy of the tree made by :meth:`widen` (plain queries; same results), 4 the 4-wide
        tree, None the mesh's tuned width."""
        opts = self._opts(band, sort, fp64_band, warps_per_block, timings, seed, radius_hint, occupancy, queue_chunk,
                          top_nodes, node_width)
        if isinstance(points, np.ndarray) and points.dtype == np.float64:
            p = np.ascontiguousarray(points).reshape(-1, 3)
            n = p.shape[0]
            d = out if out is not None else np.empty(n, np.float64)
            t = closest_tri
            check(lib.ebg_mesh_signed_distance_f64_host(self._h, _ptr(p), n, _ptr(d),
                                                        _ptr(t) if t is not None else None,
                                                        C.byref(opts), None))
            return (d, t) if t is not None else d
        if isinstance(points, np.ndarray):
            p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
            n = p.shape[0]
            d = out if out is not None else np.empty(n, np.float32)
            t = closest_tri
            check(lib.ebg_mesh_signed_distance_host(self._h, _ptr(p), n, _ptr(d),
                                                    _ptr(t) if t is not None else None,
                                                    C.byref(opts), None))
            return (d, t) if t is not None else d
        import torch
        p = points
        if p.is_cuda and p.dtype == torch.float64 and p.is_contiguous():
            n = p.numel() // 3
            d = out if out is not None else torch.empty(n, dtype=torch.float64, device=p.device)
            check(lib.ebg_mesh_signed_distance_f64(self._h, C.c_void_p(p.data_ptr()), n, C.c_void_p(d.data_ptr()),
                                                   C.c_void_p(closest_tri.data_ptr()) if closest_tri is not None
                                                   else None, C.byref(opts), _stream_ptr(stream)))
            return (d, closest_tri) if closest_tri is not None else d
        if not (p.is_cuda and p.dtype == torch.float32 and p.is_contiguous()):
            raise ValueError("points must be a contiguous float32 or float64 CUDA tensor of shape (n,3)")
        n = p.numel() // 3
        d = out if out is not None else torch.empty(n, dtype=torch.float32, device=p.device)
        check(lib.ebg_mesh_signed_distance(self._h, C.c_void_p(p.data_ptr()), n,
                                           C.c_void_p(d.data_ptr()),
                                           C.c_void_p(closest_tri.data_ptr()) if closest_tri is not None else None,
                                           C.byref(opts), _stream_ptr(stream)))
        return (d, closest_tri) if closest_tri is not None else d

    def stats(self, points, band=None, sort=True, fp64_band=True, stream=None, seed=None, radius_hint=None,
              node_width=None):
        """Traversal counters summed over the points (synchronous; CUDA tensor input)."""
        import torch
        n = points.numel() // 3
        d = torch.empty(n, dtype=torch.float32, device=points.device)
        st = _capi.QueryStats()
        opts = self._opts(band, sort, fp64_band, None, None, seed, radius_hint, node_width=node_width)
        check(lib.ebg_mesh_signed_distance_stats(self._h, C.c_void_p(points.data_ptr()), n,
                                                 C.c_void_p(d.data_ptr()), C.byref(opts),
                                                 C.byref(st), _stream_ptr(stream)))
        return d, {k: getattr(st, k) for k, _ in _capi.QueryStats._fields_}

    def check_status(self, stream=None):
        check(lib.ebg_check_status(self._h, _stream_ptr(stream)))

    def attach_seed(self, seed, cells_per_axis=0, max_entries=0, margin_cells=0.0, radius_mode=0, anchors=True,
                    stream=None):
        """Builds this mesh's per-cell entry cuts from a :class:`SeedModel` (ebg_seed_attach);
        queries passing ``seed=`` that model then start their packets from the cuts.  Returns the
        attach report as a dict.  ``radius_mode``: 0 the model's radius, 1 none, 2 exact."""
        o = _capi.AttachOpts(int(cells_per_axis), int(max_entries), float(margin_cells), int(radius_mode),
                             0 if anchors else 1)
        r = _capi.AttachReport()
        check(lib.ebg_seed_attach(self._h, seed.handle, C.byref(o), C.byref(r), _stream_ptr(stream)))
        return {k: getattr(r, k) for k, _ in _capi.AttachReport._fields_}

    def detach_seed(self):
        check(lib.ebg_seed_detach(self._h))

    def widen(self):
        """Makes the 8-wide copy of the tree (ebg_mesh_widen) that plain queries can traverse
        (``node_width=8``, or the autotuner's pick); returns {"num_nodes8", "depth8"}."""
        n8, d8 = C.c_int64(), C.c_int32()
        check(lib.ebg_mesh_widen(self._h, C.byref(n8), C.byref(d8)))
        return {"num_nodes8": n8.value, "depth8": d8.value}

    def autotune(self, sample_points, seed=None, stream=None):
        """Times the traversal launch shapes, the work-queue chunk and (plain queries of a mesh
        with an 8-wide copy, :meth:`widen`) the node width on a CUDA tensor of sample points (seeded
        with an attached :class:`SeedModel` if given) and keeps the fastest as this mesh's default;
        returns {"occupancy", "warps_per_block", "queue_chunk", "node_width", "ms"}."""
        o, w, c, nw, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_float()
        check(lib.ebg_mesh_autotune(self._h, C.c_void_p(sample_points.data_ptr()), sample_points.numel() // 3,
                                    seed.handle if seed is not None else None, C.byref(o), C.byref(w),
                                    C.byref(c), C.byref(nw), C.byref(ms), _stream_ptr(stream)))
        return {"occupancy": o.value, "warps_per_block": w.value, "queue_chunk": c.value, "node_width": nw.value,
                "ms": ms.value}


def _fp64_call(mesh, dev_fn, host_fn, points, closest_tri, stream, with_opts):
    """FP64 points (numpy: host entry, synchronous; CUDA tensor: device entry, asynchronous)."""
    opts = (C.byref(_capi.QueryOpts()),) if with_opts else ()
    t = closest_tri
    if isinstance(points, np.ndarray):
        p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        d = np.empty(p.shape[0], np.float64)
        check(host_fn(mesh._h, _ptr(p), p.shape[0], _ptr(d), _ptr(t) if t is not None else None, *opts, None))
        return (d, t) if t is not None else d
    import torch
    if not (points.is_cuda and points.dtype == torch.float64 and points.is_contiguous()):
        raise ValueError("points must be a contiguous float64 CUDA tensor of shape (n,3) or a numpy array")
    n = points.numel() // 3
    d = torch.empty(n, dtype=torch.float64, device=points.device)
    check(dev_fn(mesh._h, C.c_void_p(points.data_ptr()), n, C.c_void_p(d.data_ptr()),
                 C.c_void_p(t.data_ptr()) if t is not None else None, *opts, _stream_ptr(stream)))
    return (d, t) if t is not None else d


class MeshSDF(TriMeshSDF):
    """The reference's MeshSDF: the same mesh and tree, each triangle evaluated as a DCEL face
    (crossing-number inside test, n . (p - centroid) inside, else the nearest edge or vertex signed
    by its pseudonormal).  FP64 end to end; its values differ from TriMeshSDF's in the last bits,
    exactly as the reference's two classes do."""

    def signed_distance(self, points, closest_tri=None, stream=None):
        return _fp64_call(self, lib.ebg_mesh_signed_distance_dcel_f64, lib.ebg_mesh_signed_distance_dcel_f64_host,
                          points, closest_tri, stream, True)

    def value(self, point) -> float:
        return float(self.signed_distance(np.asarray(point, np.float64).reshape(1, 3))[0])

    signedDistance = value
    __call__ = value


def _faces_csr(faces):
    """(offsets int64, indices int32) of faces given as a list of index sequences or as an
    (offsets, indices) pair."""
    if isinstance(faces, tuple) and len(faces) == 2 and np.ndim(faces[0]) == 1 and np.ndim(faces[1]) == 1:
        return np.ascontiguousarray(faces[0], np.int64), np.ascontiguousarray(faces[1], np.int32)
    if isinstance(faces, np.ndarray) and faces.ndim == 2:
        off = np.arange(faces.shape[0] + 1, dtype=np.int64) * faces.shape[1]
        return off, np.ascontiguousarray(faces, np.int32).ravel()
    counts = np.array([len(f) for f in faces], np.int64)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    idx = np.concatenate([np.asarray(f, np.int32) for f in faces]) if len(faces) else np.empty(0, np.int32)
    return off, np.ascontiguousarray(idx, np.int32)


def polygon_normals(vertices, faces):
    """Host-only: (face normals (F,3), centroids (F,3), corner vertex normals (C,3), corner edge
    normals (C,3)) of a polygon soup, the reference's DCEL quantities (no device needed)."""
    v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
    off, idx = _faces_csr(faces)
    nf, nc = off.size - 1, idx.size
    fn, c, vn, en = np.empty((nf, 3)), np.empty((nf, 3)), np.empty((nc, 3)), np.empty((nc, 3))
    check(lib.ebg_compute_polygon_normals(_ptr(v), v.shape[0], _ptr(off), _ptr(idx), nf, _ptr(fn), _ptr(c),
                                          _ptr(vn), _ptr(en)))
    return fn, c, vn, en


class PolygonMeshSDF:
    """The reference's MeshSDF over a DCEL of polygon faces (three or more vertices each): faces
    given as a list of vertex-index sequences, an (F,k) array, or (offsets, indices).  The DCEL
    normals, the face algorithm and the smallest-|d| rule are the reference's; FP64 end to end."""

    _dev_fn = "ebg_polymesh_signed_distance"
    _host_fn = "ebg_polymesh_signed_distance_host"

    def __init__(self, vertices, faces, build="SAH", leaf_size=4, device=-1, _handle=None):
        if _handle is None:
            v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
            off, idx = _faces_csr(faces)
            b = {"SAH": BUILD_SAH, "MORTON": BUILD_MORTON}[str(build).upper()] if isinstance(build, str) else int(build)
            opts = _capi.BuildOpts(b, int(leaf_size), int(device), 0)
            _handle = C.c_void_p()
            check(lib.ebg_polymesh_create(_ptr(v), v.shape[0], _ptr(off), _ptr(idx), off.size - 1, C.byref(opts),
                                          C.byref(_handle)))
        self._h = _handle
        inf = _capi.MeshInfo()
        nc = C.c_int64()
        check(lib.ebg_polymesh_get_info(self._h, C.byref(inf), C.byref(nc)))
        self.num_faces = int(inf.num_triangles)
        self.num_corners = int(nc.value)
        self.diagonal = float(inf.diagonal)

    @classmethod
    def from_file(cls, path, build="SAH", leaf_size=4, device=-1):
        """Parser::readIntoDCEL + MeshSDF: the polygon mesh of a .stl / .obj / .ply / .vtk file."""
        b = {"SAH": BUILD_SAH, "MORTON": BUILD_MORTON}[str(build).upper()]
        opts = _capi.BuildOpts(b, int(leaf_size), int(device), 0)
        h = C.c_void_p()
        check(lib.ebg_polymesh_create_from_file(str(path).encode(), C.byref(opts), C.byref(h)))
        return cls(None, None, _handle=h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.ebg_polymesh_destroy(h)
            self._h = None

    def normals(self):
        """(face normals (F,3), centroids (F,3), corner vertex normals (C,3), corner edge normals
        (C,3)), corners face after face in soup order."""
        fn, c = np.empty((self.num_faces, 3)), np.empty((self.num_faces, 3))
        vn, en = np.empty((self.num_corners, 3)), np.empty((self.num_corners, 3))
        check(lib.ebg_polymesh_get_normals(self._h, _ptr(fn), _ptr(c), _ptr(vn), _ptr(en)))
        return fn, c, vn, en

    def signed_distance(self, points, closest_face=None, stream=None):
        """FP64 signed distances (numpy: synchronous host call; CUDA float64 tensor: asynchronous)."""
        return _fp64_call(self, getattr(lib, self._dev_fn), getattr(lib, self._host_fn), points, closest_face,
                          stream, False)

    def check_status(self, stream=None):
        check(lib.ebg_polymesh_check_status(self._h, _stream_ptr(stream)))

    def value(self, point) -> float:
        return float(self.signed_distance(np.asarray(point, np.float64).reshape(1, 3))[0])

    signedDistance = value
    __call__ = value


class PolygonFlatMeshSDF(PolygonMeshSDF):
    """The reference's FlatMeshSDF over polygon faces: every face for every point, the first face
    in soup order with the smallest unsigned distance."""

    _dev_fn = "ebg_polymesh_signed_distance_flat"
    _host_fn = "ebg_polymesh_signed_distance_flat_host"


class FlatMeshSDF(TriMeshSDF):
    """The reference's FlatMeshSDF: no tree search; every triangle for every point (DCEL face
    algorithm, the first triangle in soup order with the smallest unsigned distance wins).
    O(points x triangles), FP64: a ground truth for small meshes."""

    def signed_distance(self, points, closest_tri=None, stream=None):
        return _fp64_call(self, lib.ebg_mesh_signed_distance_flat_f64, lib.ebg_mesh_signed_distance_flat_f64_host,
                          points, closest_tri, stream, False)

    def value(self, point) -> float:
        return float(self.signed_distance(np.asarray(point, np.float64).reshape(1, 3))[0])

    signedDistance = value
    __call__ = value


class PointCloudBVH:
    """k-nearest-neighbour search over a point cloud (the reference's PointCloudBVH).

    ``points``: (n,3) float32, a numpy array (built after a host->device copy) or a CUDA tensor
    (built in place).  Neighbours come in increasing (squared distance, index) order, so equal
    distances resolve to the lowest index; squared distances are the reference's float arithmetic.
    ``leaf_size``: at most that many points per leaf (<= 32).  The tree divides the Morton-ordered
    points where the Morton curve jumps; ``balanced=True`` groups fixed runs of ``leaf_size`` points
    four at a time instead (the same answers, more work per query on clustered clouds).
    """

    def __init__(self, points, leaf_size=8, device=-1, stream=None, balanced=False):
        opts = _capi.BuildOpts(0, int(leaf_size), int(device), 2 if balanced else 0)
        h = C.c_void_p()
        if isinstance(points, np.ndarray):
            p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
            check(lib.ebg_cloud_create(_ptr(p), p.shape[0], C.byref(opts), C.byref(h)))
            self.n = p.shape[0]
        else:
            import torch
            if not (points.is_cuda and points.dtype == torch.float32 and points.is_contiguous()):
                raise ValueError("points must be a contiguous float32 CUDA tensor of shape (n,3)")
            self.n = points.numel() // 3
            check(lib.ebg_cloud_create_device(C.c_void_p(points.data_ptr()), self.n, C.byref(opts), C.byref(h),
                                              _stream_ptr(stream)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.ebg_cloud_destroy(h)
            self._h = None

    def tree_info(self):
        """{"nodes": 4-wide nodes, "depth": node levels, "radix": False for the balanced tree}."""
        nn, d, r = C.c_int64(), C.c_int32(), C.c_int32()
        check(lib.ebg_cloud_tree_info(self._h, C.byref(nn), C.byref(d), C.byref(r)))
        return {"nodes": nn.value, "depth": d.value, "radix": bool(r.value)}

    def numPoints(self) -> int:
        return int(lib.ebg_cloud_size(self._h))

    def knn(self, queries, k, sort=True, stream=None):
        """(idx (nq,k) int32, d2 (nq,k) float32) for (nq,3) float32 queries (CUDA tensor: asynchronous
        on ``stream``; numpy: synchronous host call)."""
        opts = _capi.QueryOpts(0.0, 0 if sort else 1, 0, None, 0, 0, None)
        if isinstance(queries, np.ndarray):
            q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 3)
            idx = np.empty((q.shape[0], k), np.int32)
            d2 = np.empty((q.shape[0], k), np.float32)
            check(lib.ebg_cloud_knn_host(self._h, _ptr(q), q.shape[0], int(k), _ptr(idx), _ptr(d2), C.byref(opts),
                                         None))
            return idx, d2
        import torch
        if not (queries.is_cuda and queries.dtype == torch.float32 and queries.is_contiguous()):
            raise ValueError("queries must be a contiguous float32 CUDA tensor of shape (n,3)")
        nq = queries.numel() // 3
        idx = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        d2 = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
        check(lib.ebg_cloud_knn(self._h, C.c_void_p(queries.data_ptr()), nq, int(k), C.c_void_p(idx.data_ptr()),
                                C.c_void_p(d2.data_ptr()), C.byref(opts), _stream_ptr(stream)))
        return idx, d2

    # --- the reference's single-point API (PointCloudBVHImplem.hpp:429-453) -----------------------
    def closestPoint(self, q):
        """(index, squared distance) of the nearest point."""
        idx, d2 = self.knn(np.asarray(q, np.float32).reshape(1, 3), 1)
        return int(idx[0, 0]), float(d2[0, 0])

    def closestPoints(self, q, k):
        """The k nearest as a list of (index, squared distance), nearest first."""
        idx, d2 = self.knn(np.asarray(q, np.float32).reshape(1, 3), k)
        return [(int(i), float(d)) for i, d in zip(idx[0], d2[0]) if i >= 0]

    # --- self queries (PointCloudBVHImplem.hpp:455-507): the point itself is excluded -------------
    def all_nearest_neighbors(self, k=1, device=False, stream=None):
        """allNearestNeighbors: (idx (n,k) int32, d2 (n,k) float32), row i = the k nearest other
        points of cloud point i, in (d2, index) order.  device=True returns CUDA tensors
        (asynchronous on ``stream``)."""
        if not device:
            idx = np.empty((self.n, k), np.int32)
            d2 = np.empty((self.n, k), np.float32)
            check(lib.ebg_cloud_self_knn_host(self._h, int(k), _ptr(idx), _ptr(d2), None))
            return idx, d2
        import torch
        idx = torch.empty((self.n, k), dtype=torch.int32, device="cuda")
        d2 = torch.empty((self.n, k), dtype=torch.float32, device="cuda")
        check(lib.ebg_cloud_self_knn(self._h, int(k), C.c_void_p(idx.data_ptr()), C.c_void_p(d2.data_ptr()),
                                     _stream_ptr(stream)))
        return idx, d2

    allNearestNeighbors = all_nearest_neighbors

    def nearest_neighbors(self, point_ids, k=1, stream=None):
        """nearestNeighbors(point, k) for a list of cloud indices (CUDA int64 tensor, or anything
        numpy can turn into int64: then the call synchronises and returns numpy arrays)."""
        import torch
        host = not (isinstance(point_ids, torch.Tensor) and point_ids.is_cuda)
        ids = torch.as_tensor(np.asarray(point_ids, np.int64) if host else point_ids, dtype=torch.int64).cuda()
        ids = ids.contiguous().reshape(-1)
        m = ids.numel()
        idx = torch.empty((m, k), dtype=torch.int32, device=ids.device)
        d2 = torch.empty((m, k), dtype=torch.float32, device=ids.device)
        check(lib.ebg_cloud_self_knn_points(self._h, C.c_void_p(ids.data_ptr()), m, int(k),
                                            C.c_void_p(idx.data_ptr()), C.c_void_p(d2.data_ptr()),
                                            _stream_ptr(stream)))
        if host:
            self.check_status(stream)
            return idx.cpu().numpy(), d2.cpu().numpy()
        return idx, d2

    def nearestNeighbor(self, point_id):
        """(index, squared distance) of the nearest other point of cloud point ``point_id``."""
        idx, d2 = self.nearest_neighbors([int(point_id)], 1)
        return int(idx[0, 0]), float(d2[0, 0])

    def check_status(self, stream=None):
        check(lib.ebg_cloud_check_status(self._h, _stream_ptr(stream)))


class PointCloudHashGrid:
    """k-nearest-neighbour search over a point cloud on a uniform grid (the reference's
    PointCloudHashGrid), with PointCloudBVH's interface and results.

    ``points``: (n,3) float32 numpy array (n may be 0).  ``target_per_cell`` sets the cell size as
    the reference does: cells hold that many points at the cloud's average density.  Neighbours
    come in increasing (squared distance, index) order -- equal distances resolve to the lowest
    index -- so the answers equal :class:`PointCloudBVH`'s.
    """

    def __init__(self, points, target_per_cell=1.0, device=-1):
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        h = C.c_void_p()
        check(lib.ebg_grid_create(_ptr(p) if p.size else None, p.shape[0], float(target_per_cell), int(device),
                                  C.byref(h)))
        self._h = h
        self.n = p.shape[0]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.ebg_grid_destroy(h)
            self._h = None

    def numPoints(self) -> int:
        return int(lib.ebg_grid_size(self._h))

    def grid_info(self):
        """((cells x, y, z), cell size)."""
        cells = (C.c_int32 * 3)()
        h = C.c_double()
        check(lib.ebg_grid_info(self._h, cells, C.byref(h)))
        return tuple(cells), h.value

    def knn(self, queries, k, stream=None):
        """(idx (nq,k) int32, d2 (nq,k) float32) for (nq,3) float32 queries (CUDA tensor: asynchronous
        on ``stream``; numpy: synchronous host call)."""
        if isinstance(queries, np.ndarray):
            q = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, 3)
            idx = np.empty((q.shape[0], k), np.int32)
            d2 = np.empty((q.shape[0], k), np.float32)
            check(lib.ebg_grid_knn_host(self._h, _ptr(q), q.shape[0], int(k), _ptr(idx), _ptr(d2), None))
            return idx, d2
        import torch
        if not (queries.is_cuda and queries.dtype == torch.float32 and queries.is_contiguous()):
            raise ValueError("queries must be a contiguous float32 CUDA tensor of shape (n,3)")
        nq = queries.numel() // 3
        idx = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        d2 = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
        check(lib.ebg_grid_knn(self._h, C.c_void_p(queries.data_ptr()), nq, int(k), C.c_void_p(idx.data_ptr()),
                               C.c_void_p(d2.data_ptr()), _stream_ptr(stream)))
        return idx, d2

    # --- the reference's single-point API (PointCloudHashGridImplem.hpp:309-333) -----------------
    def closestPoint(self, q):
        """(index, squared distance) of the nearest point; (-1, inf) for an empty cloud."""
        idx, d2 = self.knn(np.asarray(q, np.float32).reshape(1, 3), 1)
        return int(idx[0, 0]), float(d2[0, 0])

    def closestPoints(self, q, k):
        """The k nearest as a list of (index, squared distance), nearest first."""
        idx, d2 = self.knn(np.asarray(q, np.float32).reshape(1, 3), k)
        return [(int(i), float(d)) for i, d in zip(idx[0], d2[0]) if i >= 0]

    # --- self queries (PointCloudHashGridImplem.hpp:335-385): the point itself is excluded --------
    def all_nearest_neighbors(self, k=1, device=False, stream=None):
        """allNearestNeighbors: (idx (n,k) int32, d2 (n,k) float32), row i = the k nearest other
        points of cloud point i.  device=True returns CUDA tensors (asynchronous on ``stream``)."""
        if not device:
            idx = np.empty((self.n, k), np.int32)
            d2 = np.empty((self.n, k), np.float32)
            check(lib.ebg_grid_self_knn_host(self._h, int(k), _ptr(idx), _ptr(d2), None))
            return idx, d2
        import torch
        idx = torch.empty((self.n, k), dtype=torch.int32, device="cuda")
        d2 = torch.empty((self.n, k), dtype=torch.float32, device="cuda")
        check(lib.ebg_grid_self_knn(self._h, int(k), C.c_void_p(idx.data_ptr()), C.c_void_p(d2.data_ptr()),
                                    _stream_ptr(stream)))
        return idx, d2

    allNearestNeighbors = all_nearest_neighbors

    def nearest_neighbors(self, point_ids, k=1):
        """nearestNeighbors(point, k) for a list of cloud indices; synchronous, numpy results."""
        ids = np.ascontiguousarray(np.asarray(point_ids, np.int64).reshape(-1))
        idx = np.empty((ids.size, k), np.int32)
        d2 = np.empty((ids.size, k), np.float32)
        check(lib.ebg_grid_self_knn_points_host(self._h, _ptr(ids), ids.size, int(k), _ptr(idx), _ptr(d2), None))
        return idx, d2

    def nearestNeighbor(self, point_id):
        """(index, squared distance) of the nearest other point of cloud point ``point_id``."""
        idx, d2 = self.nearest_neighbors([int(point_id)], 1)
        return int(idx[0, 0]), float(d2[0, 0])

    def check_status(self, stream=None):
        check(lib.ebg_grid_check_status(self._h, _stream_ptr(stream)))


class SeedModel:
    """Learned pruning radius for :class:`TriMeshSDF` queries (no counterpart in the reference).

    A 16-level hash-grid encoding with a 3-layer, 64-wide BF16 ReLU MLP, trained on the GPU by the
    library's own kernels on exact signed distances the mesh path generates.  Attach it to a mesh
    (``mesh.attach_seed(model)``, done by :meth:`train`), then query with
    ``mesh.signed_distance(points, seed=model)``.
    """

    def __init__(self, handle):
        self._h = handle

    @staticmethod
    def _opts(**kw):
        o = _capi.SeedOpts()
        for k, v in kw.items():
            if k in ("lo", "hi"):
                getattr(o, k)[:] = [float(x) for x in v]
            elif v is not None:
                setattr(o, k, v)
        return o

    @classmethod
    def train(cls, mesh, stream=None, attach=True, **kw):
        """Trains on ``mesh`` (see ebg_seed_opts for the keyword options) and, unless ``attach`` is
        False, attaches the model to it with the default cells (:meth:`TriMeshSDF.attach_seed`)."""
        o = cls._opts(**kw)
        h = C.c_void_p()
        rep = _capi.SeedReport()
        check(lib.ebg_seed_train(mesh.handle, C.byref(o), C.byref(h), C.byref(rep),
                                 _stream_ptr(stream) if stream is not None else None))
        model = cls(h)
        if attach:
            mesh.attach_seed(model, stream=stream)
        return model

    @classmethod
    def create(cls, **kw):
        """Untrained model (random parameters) over the domain lo..hi."""
        o = cls._opts(**kw)
        h = C.c_void_p()
        check(lib.ebg_seed_create(C.byref(o), C.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path, device=-1):
        h = C.c_void_p()
        check(lib.ebg_seed_load(str(path).encode(), int(device), C.byref(h)))
        return cls(h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.ebg_seed_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def report(self):
        r = _capi.SeedReport()
        check(lib.ebg_seed_get_report(self._h, C.byref(r)))
        return {k: getattr(r, k) for k, _ in _capi.SeedReport._fields_}

    def save(self, path):
        check(lib.ebg_seed_save(self._h, str(path).encode()))

    def predict(self, points, stream=None):
        """Raw predicted signed distance at (n,3) float32 CUDA points."""
        import torch
        n = points.numel() // 3
        out = torch.empty(n, dtype=torch.float32, device=points.device)
        check(lib.ebg_seed_predict(self._h, C.c_void_p(points.data_ptr()), n, C.c_void_p(out.data_ptr()),
                                   _stream_ptr(stream)))
        return out

    def get_params(self, table_size):
        table = np.empty(table_size, np.float32)
        params = np.empty(10497, np.float32)
        check(lib.ebg_seed_get_params(self._h, _ptr(table), _ptr(params)))
        return table, params

    def set_params(self, table=None, params=None):
        t = np.ascontiguousarray(table, np.float32) if table is not None else None
        p = np.ascontiguousarray(params, np.float32) if params is not None else None
        check(lib.ebg_seed_set_params(self._h, _ptr(t) if t is not None else None,
                                      _ptr(p) if p is not None else None))

    def gradients(self, points, targets, eps, table_size):
        """(loss, grad_table, grad_params) of one batch, parameters unchanged."""
        import torch
        pt = torch.from_numpy(np.ascontiguousarray(points, np.float32)).cuda()
        tt = torch.from_numpy(np.ascontiguousarray(targets, np.float32)).cuda()
        loss = C.c_float()
        gt = np.empty(table_size, np.float32)
        gp = np.empty(10497, np.float32)
        check(lib.ebg_seed_gradients(self._h, C.c_void_p(pt.data_ptr()), C.c_void_p(tt.data_ptr()),
                                     pt.shape[0], float(eps), C.byref(loss), _ptr(gt), _ptr(gp)))
        return loss.value, gt, gp


class BVHUnion:
    """Union of spheres and posed mesh instances (the reference's BVHUnionIF over SphereSDF and
    Translate(Rotate(TriMeshSDF)) objects).  ``spheres``: (S,4) centre xyz + radius; ``meshes``:
    list of :class:`TriMeshSDF`; ``poses``: (M,5) angle in degrees, axis (0/1/2), translation."""

    def __init__(self, spheres=None, meshes=(), poses=None, leaf_size=3, device=-1):
        sp = np.ascontiguousarray(spheres if spheres is not None else np.zeros((0, 4)), np.float64).reshape(-1, 4)
        ps = np.ascontiguousarray(poses if poses is not None else np.zeros((0, 5)), np.float64).reshape(-1, 5)
        self._meshes = list(meshes)  # kept alive: the scene references their device data
        arr = (C.c_void_p * max(1, len(self._meshes)))(*[m.handle.value for m in self._meshes])
        opts = _capi.BuildOpts(0, int(leaf_size), int(device), 0)
        h = C.c_void_p()
        check(lib.ebg_scene_create(sp.shape[0], _ptr(sp), len(self._meshes), arr, _ptr(ps), C.byref(opts),
                                   C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.ebg_scene_destroy(h)
            self._h = None

    def num_objects(self) -> int:
        return int(lib.ebg_scene_num_objects(self._h))

    def values(self, points, out=None, sort=True, fp64_band=True, stream=None):
        """Union value at (n,3) float32 points (CUDA tensor: asynchronous; numpy: synchronous)."""
        opts = _capi.QueryOpts(0.0, 0 if sort else 1, 0 if fp64_band else 1, None, 0, 0, None)
        if isinstance(points, np.ndarray):
            p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
            d = out if out is not None else np.empty(p.shape[0], np.float32)
            check(lib.ebg_scene_value_host(self._h, _ptr(p), p.shape[0], _ptr(d), C.byref(opts), None))
            return d
        import torch
        n = points.numel() // 3
        d = out if out is not None else torch.empty(n, dtype=torch.float32, device=points.device)
        check(lib.ebg_scene_value(self._h, C.c_void_p(points.data_ptr()), n, C.c_void_p(d.data_ptr()),
                                  C.byref(opts), _stream_ptr(stream)))
        return d

    def value(self, point) -> float:
        return float(self.values(np.asarray(point, np.float32).reshape(1, 3))[0])

    def values_batches(self, batches, outs=None, sort=True, fp64_band=True, stream=None):
        """Union values of several batches of (n_i,3) float32 CUDA points in one call
        (ebg_scene_eval_batches: one persistent launch for all of them).  Returns the list of
        result tensors (``outs`` if given).  Asynchronous on ``stream``."""
        import torch
        if not batches:
            return []
        dev = batches[0].device
        outs = outs if outs is not None else [torch.empty(b.numel() // 3, dtype=torch.float32, device=dev)
                                              for b in batches]
        desc = np.zeros((len(batches), 3), np.int64)  # ebg_batch: points, n, out
        for i, (b, o) in enumerate(zip(batches, outs)):
            if not (b.is_cuda and b.dtype == torch.float32 and b.is_contiguous()):
                raise ValueError("batches must be contiguous float32 CUDA tensors of shape (n,3)")
            desc[i] = (b.data_ptr(), b.numel() // 3, o.data_ptr())
        # the descriptors live on the device and must outlive the asynchronous call; the same
        # batches again reuse them (no host-to-device copy, so such a call can be graph-captured)
        key = desc.tobytes()
        if getattr(self, "_batch_key", None) != key:
            self._batch_desc = torch.from_numpy(desc).to(dev, non_blocking=False)
            self._batch_key = key
        d = self._batch_desc
        opts = _capi.QueryOpts(0.0, 0 if sort else 1, 0 if fp64_band else 1, None, 0, 0, None)
        check(lib.ebg_scene_eval_batches(self._h, C.c_void_p(d.data_ptr()), len(batches), int(desc[:, 1].sum()),
                                         C.byref(opts), _stream_ptr(stream)))
        return outs

    def autotune(self, sample_points, stream=None):
        """Times the work-queue chunk on a CUDA tensor of sample points and keeps the fastest as
        this scene's default; returns {"queue_chunk", "ms"}."""
        c, ms = C.c_int32(), C.c_float()
        check(lib.ebg_scene_autotune(self._h, C.c_void_p(sample_points.data_ptr()), sample_points.numel() // 3,
                                     C.byref(c), C.byref(ms), _stream_ptr(stream)))
        return {"queue_chunk": c.value, "ms": ms.value}

    def check_status(self, stream=None):
        check(lib.ebg_scene_check_status(self._h, _stream_ptr(stream)))
