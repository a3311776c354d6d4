"""ORACLE -- test infrastructure, not the product.

Loads the two CPU oracles built by ``oracle/Makefile``:

* ``ref()``  -- the UNMODIFIED reference library (rmrsk/EBGeometry, header-only C++17) compiled
  from its own headers with the extern "C" batch wrappers of ``ref_harness.cpp``
  (``oracle/_ref/libebgref_{avx512,avx2}.so``; the variant matching the host CPU is loaded).
* ``port()`` -- the plain-C restatement ``ebg_port.c`` (``oracle/_port/libebgport.so``).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg / reference arm may import
this package, and only as the checker or as the timed CPU baseline -- never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_LIB = os.path.join(HERE, "_port", "libebgport.so")

_P = C.c_void_p
_I64 = C.c_int64
_D = C.c_double


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    fl = line.split()
                    return all(f in fl for f in ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512cd"))
    except OSError:
        pass
    return False


def _cpu_flags():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    return set(line.split())
    except OSError:
        pass
    return set()


def ref_lib_path(timing: bool = False) -> str:
    """The reference oracle's library: the parity build (no fused multiply-adds), or with ``timing``
    the -O3 -march=sapphirerapids build with fused multiply-adds, where the host supports it."""
    if timing and {"avx512_fp16", "amx_tile", "avx512_bf16"} <= _cpu_flags():
        fast = os.path.join(REF_DIR, "libebgref_fast.so")
        if os.path.exists(fast):
            return fast
    name = "libebgref_avx512.so" if _cpu_has_avx512() else "libebgref_avx2.so"
    return os.path.join(REF_DIR, name)


_SOURCE_NOTE = os.path.join(REF_DIR, "source_dir.txt")


def reference_dir():
    """Directory of the reference sources: EBG_REFERENCE_DIR, else the one the reference oracle was
    last built from (recorded beside it); None when neither names an existing directory."""
    d = os.environ.get("EBG_REFERENCE_DIR")
    if not d and os.path.exists(_SOURCE_NOTE):
        with open(_SOURCE_NOTE) as fh:
            d = fh.read().strip()
    return d if d and os.path.isdir(d) else None


def build(reference_dir: str | None = None, quiet: bool = True) -> None:
    """Builds the port and, when the reference sources are given (argument or EBG_REFERENCE_DIR)
    and present, the reference oracle."""
    ref = reference_dir or os.environ.get("EBG_REFERENCE_DIR")
    targets = ["port"]
    if ref and os.path.isdir(ref):
        targets.append("ref")
    subprocess.run(["make", "-C", HERE, *([f"REF={ref}"] if "ref" in targets else []), *targets], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
    if "ref" in targets:
        with open(_SOURCE_NOTE, "w") as fh:
            fh.write(os.path.abspath(ref) + "\n")


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class _Ref:
    def __init__(self, path):
        lib = C.CDLL(path)
        sig = {
            "ref_omp_max_threads": (C.c_int, []),
            "ref_mesh_create": (_P, [_P, _I64, _P, _I64, C.c_int, C.c_int, C.c_int]),
            "ref_polymesh_create": (_P, [_P, _I64, _P, _P, _I64, C.c_int]),
            "ref_polymesh_normals": (C.c_int, [_P, _P, _P, _P, _P]),
            "ref_read_polysoup": (C.c_int, [C.c_char_p, _P, _P, _P, _P, _P, _P]),
            "ref_mesh_destroy": (None, [_P]),
            "ref_mesh_sdf": (C.c_int, [_P, _P, _I64, _P, C.c_int, C.c_int]),
            "ref_mesh_value1": (_D, [_P, _D, _D, _D]),
            "ref_mesh_face_normals": (C.c_int, [_P, _P, _P, _P]),
            "ref_triangle_sd": (_D, [_P, _P, _P, _P]),
            "ref_trisoa4_sd": (_D, [C.c_int, _P, _P, _P, _P]),
            "ref_read_soup": (C.c_int, [C.c_char_p, _P, C.POINTER(_I64), _P, C.POINTER(_I64)]),
            "ref_sample_points": (None, [_I64, C.c_uint64, _P]),
            "ref_make_cloud_mt19937": (None, [_I64, C.c_uint32, _P]),
            "ref_cloud_create": (_P, [_P, _I64]),
            "ref_cloud_destroy": (None, [_P]),
            "ref_cloud_knn": (C.c_int, [_P, _P, _I64, C.c_int, _P, _P, C.c_int]),
            "ref_cloud_knn_lex": (C.c_int, [_P, _P, _I64, C.c_int, _P, _P, C.c_int]),
            "ref_cloud_knn_lex_excl": (C.c_int, [_P, _P, _I64, C.c_int, _P, _P, C.c_int, C.c_int]),
            "ref_cloud_all_nn": (C.c_int, [_P, C.c_int, _I64, _P, _P]),
            "ref_grid_create": (_P, [_P, _I64, C.c_float]),
            "ref_grid_destroy": (None, [_P]),
            "ref_grid_knn": (C.c_int, [_P, _P, _P, _I64, C.c_int, _P, _P, C.c_int]),
            "ref_grid_all_nn": (C.c_int, [_P, C.c_int, _I64, _P, _P]),
            "ref_scene_create": (_P, [_I64, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P]),
            "ref_scene_destroy": (None, [_P]),
            "ref_scene_value": (C.c_int, [_P, _P, _I64, _P, C.c_int, C.c_int]),
        }
        for k, (r, a) in sig.items():
            fn = getattr(lib, k)
            fn.restype = r
            fn.argtypes = a
        self.lib = lib
        self.path = path

    def max_threads(self) -> int:
        return int(self.lib.ref_omp_max_threads())

    # meshes ------------------------------------------------------------------------------------
    class Mesh:
        """Reference TriMeshSDF built through Soup::soupToDCEL.  kind 0: <double,short,4,4>;
        kind 1: ISA-default K/W; kind 3: MeshSDF<double,short,4> over the DCEL faces.  build 0 SAH,
        1 Morton."""

        def __init__(self, ref, v, f, kind=0, build=0, max_leaf_groups=4):
            self.ref = ref
            self.v = np.ascontiguousarray(v, np.float64)
            self.f = np.ascontiguousarray(f, np.int64)
            self.h = ref.lib.ref_mesh_create(_ptr(self.v), self.v.shape[0], _ptr(self.f), self.f.shape[0],
                                             kind, build, max_leaf_groups)

        def __del__(self):
            if getattr(self, "h", None):
                self.ref.lib.ref_mesh_destroy(self.h)
                self.h = None

        def sdf(self, p, flat=False, threads=0, dcel=False):
            """flat: FlatMeshSDF (DCEL faces, brute force); dcel: the MeshSDF (needs kind 3)."""
            p = np.ascontiguousarray(p, np.float64).reshape(-1, 3)
            out = np.empty(p.shape[0])
            which = 1 if flat else (2 if dcel else 0)
            rc = self.ref.lib.ref_mesh_sdf(self.h, _ptr(p), p.shape[0], _ptr(out), which, threads)
            assert rc == 0
            return out

        def normals(self):
            t = self.f.shape[0]
            fn, vn, en = np.empty((t, 3)), np.empty((t, 3, 3)), np.empty((t, 3, 3))
            self.ref.lib.ref_mesh_face_normals(self.h, _ptr(fn), _ptr(vn), _ptr(en))
            return fn, vn, en

    def mesh(self, v, f, kind=0, build=0, max_leaf_groups=4):
        return _Ref.Mesh(self, v, f, kind, build, max_leaf_groups)

    class PolyMesh(Mesh):
        """Reference MeshSDF<double,short,4> and FlatMeshSDF over a polygon soup (faces: offsets,
        indices).  sdf(p, dcel=True) is the MeshSDF, sdf(p, flat=True) the FlatMeshSDF."""

        def __init__(self, ref, v, off, idx, build=0):
            self.ref = ref
            self.v = np.ascontiguousarray(v, np.float64)
            self.off = np.ascontiguousarray(off, np.int64)
            self.idx = np.ascontiguousarray(idx, np.int64)
            self.h = ref.lib.ref_polymesh_create(_ptr(self.v), self.v.shape[0], _ptr(self.off), _ptr(self.idx),
                                                 self.off.size - 1, build)

        def polygon_normals(self):
            nf, nc = self.off.size - 1, self.idx.size
            fn, c, vn, en = np.empty((nf, 3)), np.empty((nf, 3)), np.empty((nc, 3)), np.empty((nc, 3))
            assert self.ref.lib.ref_polymesh_normals(self.h, _ptr(fn), _ptr(c), _ptr(vn), _ptr(en)) == 0
            return fn, c, vn, en

    def polymesh(self, v, off, idx, build=0):
        return _Ref.PolyMesh(self, v, off, idx, build)

    def read_polysoup(self, path):
        nv, nf, nc = (C.c_int64(), C.c_int64(), C.c_int64())
        assert self.lib.ref_read_polysoup(str(path).encode(), None, C.byref(nv), None, None, C.byref(nf),
                                          C.byref(nc)) == 0
        v = np.empty((nv.value, 3))
        off = np.empty(nf.value + 1, np.int64)
        idx = np.empty(nc.value, np.int64)
        assert self.lib.ref_read_polysoup(str(path).encode(), _ptr(v), C.byref(nv), _ptr(off), _ptr(idx),
                                          C.byref(nf), C.byref(nc)) == 0
        return v, off, idx

    def triangle_sd(self, v, vn, en, p) -> float:
        a = [np.ascontiguousarray(x, np.float64).ravel() for x in (v, vn, en, p)]
        return float(self.lib.ref_triangle_sd(*[_ptr(x) for x in a]))

    def trisoa4_sd(self, v, vn, en, p) -> float:
        v = np.ascontiguousarray(v, np.float64).reshape(-1, 9)
        a = [v, np.ascontiguousarray(vn, np.float64).reshape(-1, 9),
             np.ascontiguousarray(en, np.float64).reshape(-1, 9), np.ascontiguousarray(p, np.float64)]
        return float(self.lib.ref_trisoa4_sd(v.shape[0], *[_ptr(x) for x in a]))

    def read_soup(self, path):
        nv, nf = _I64(), _I64()
        rc = self.lib.ref_read_soup(path.encode(), None, C.byref(nv), None, C.byref(nf))
        assert rc == 0, rc
        v = np.empty((nv.value, 3))
        f = np.empty((nf.value, 3), np.int64)
        rc = self.lib.ref_read_soup(path.encode(), _ptr(v), C.byref(nv), _ptr(f), C.byref(nf))
        assert rc == 0, rc
        return v, f

    def sample_points(self, n, seed):
        out = np.empty((n, 3))
        self.lib.ref_sample_points(n, seed, _ptr(out))
        return out

    def make_cloud_mt19937(self, n, seed):
        out = np.empty((n, 3), np.float32)
        self.lib.ref_make_cloud_mt19937(n, seed, _ptr(out))
        return out

    # point clouds --------------------------------------------------------------------------------
    class Cloud:
        def __init__(self, ref, p):
            self.ref = ref
            self.p = np.ascontiguousarray(p, np.float32).reshape(-1, 3)
            self.h = ref.lib.ref_cloud_create(_ptr(self.p), self.p.shape[0])

        def __del__(self):
            if getattr(self, "h", None):
                self.ref.lib.ref_cloud_destroy(self.h)
                self.h = None

        def knn(self, q, k, lex=True, threads=0):
            q = np.ascontiguousarray(q, np.float32).reshape(-1, 3)
            idx = np.empty((q.shape[0], k), np.int64)
            d2 = np.empty((q.shape[0], k), np.float32)
            fn = self.ref.lib.ref_cloud_knn_lex if lex else self.ref.lib.ref_cloud_knn
            assert fn(self.h, _ptr(q), q.shape[0], k, _ptr(idx), _ptr(d2), threads) == 0
            return idx, d2

        def self_knn(self, k, lex=True, threads=0):
            """Every cloud point's k neighbours, itself excluded.  lex: the reference's traversal
            with a (d2, index) state (lowest index on ties); else its own allNearestNeighbors."""
            n = self.p.shape[0]
            idx = np.empty((n, k), np.int64)
            d2 = np.empty((n, k), np.float32)
            if lex:
                rc = self.ref.lib.ref_cloud_knn_lex_excl(self.h, _ptr(self.p), n, k, _ptr(idx), _ptr(d2), threads, 1)
            else:
                rc = self.ref.lib.ref_cloud_all_nn(self.h, k, n, _ptr(idx), _ptr(d2))
            assert rc == 0
            return idx, d2

    def cloud(self, p):
        return _Ref.Cloud(self, p)

    class Grid:
        """The reference's PointCloudHashGrid<float> (its own tie order: visiting order)."""

        def __init__(self, ref, p, target=1.0):
            self.ref = ref
            self.p = np.ascontiguousarray(p, np.float32).reshape(-1, 3)
            self.h = ref.lib.ref_grid_create(_ptr(self.p) if self.p.size else None, self.p.shape[0], float(target))

        def __del__(self):
            if getattr(self, "h", None):
                self.ref.lib.ref_grid_destroy(self.h)
                self.h = None

        def knn(self, q, k, threads=0):
            q = np.ascontiguousarray(q, np.float32).reshape(-1, 3)
            idx = np.empty((q.shape[0], k), np.int64)
            d2 = np.empty((q.shape[0], k), np.float32)
            assert self.ref.lib.ref_grid_knn(self.h, _ptr(q), None, q.shape[0], k, _ptr(idx), _ptr(d2), threads) == 0
            return idx, d2

        def nearest_neighbors(self, ids, k, threads=0):
            ids = np.ascontiguousarray(ids, np.int64).reshape(-1)
            idx = np.empty((ids.size, k), np.int64)
            d2 = np.empty((ids.size, k), np.float32)
            assert self.ref.lib.ref_grid_knn(self.h, None, _ptr(ids), ids.size, k, _ptr(idx), _ptr(d2), threads) == 0
            return idx, d2

        def all_nn(self, k):
            n = self.p.shape[0]
            idx = np.empty((n, k), np.int64)
            d2 = np.empty((n, k), np.float32)
            assert self.ref.lib.ref_grid_all_nn(self.h, k, n, _ptr(idx), _ptr(d2)) == 0
            return idx, d2

    def grid(self, p, target=1.0):
        return _Ref.Grid(self, p, target)

    # CSG -----------------------------------------------------------------------------------------
    class Scene:
        def __init__(self, ref, spheres, meshes, poses, bboxes):
            self.ref = ref
            self.spheres = np.ascontiguousarray(spheres, np.float64).reshape(-1, 4)
            vs = [np.asarray(v, np.float64) for v, _ in meshes]
            fs = [np.asarray(f, np.int64) for _, f in meshes]
            self.V = np.ascontiguousarray(np.concatenate(vs) if vs else np.zeros((0, 3)))
            self.F = np.ascontiguousarray(np.concatenate(fs) if fs else np.zeros((0, 3), np.int64))
            self.vcnt = np.array([v.shape[0] for v in vs], np.int64)
            self.fcnt = np.array([f.shape[0] for f in fs], np.int64)
            self.voff = np.concatenate([[0], np.cumsum(self.vcnt)[:-1]]).astype(np.int64)
            self.foff = np.concatenate([[0], np.cumsum(self.fcnt)[:-1]]).astype(np.int64)
            self.poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 5)
            self.bboxes = np.ascontiguousarray(bboxes, np.float64).reshape(-1, 6)
            self.h = ref.lib.ref_scene_create(self.spheres.shape[0], _ptr(self.spheres), len(meshes), _ptr(self.V),
                                              _ptr(self.voff), _ptr(self.vcnt), _ptr(self.F), _ptr(self.foff),
                                              _ptr(self.fcnt), _ptr(self.poses), _ptr(self.bboxes))

        def __del__(self):
            if getattr(self, "h", None):
                self.ref.lib.ref_scene_destroy(self.h)
                self.h = None

        def value(self, p, brute=False, threads=0):
            p = np.ascontiguousarray(p, np.float64).reshape(-1, 3)
            out = np.empty(p.shape[0])
            assert self.ref.lib.ref_scene_value(self.h, _ptr(p), p.shape[0], _ptr(out), int(brute), threads) == 0
            return out

    def scene(self, spheres, meshes, poses, bboxes):
        return _Ref.Scene(self, spheres, meshes, poses, bboxes)


class _Port:
    def __init__(self, path):
        lib = C.CDLL(path)
        sig = {
            "port_triangle_sd": (_D, [_P, _P, _P, _P, _P]),
            "port_triangle_sd_scalar": (_D, [_P, _P, _P, _P, _P]),
            "port_mesh_normals": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _P]),
            "port_mesh_sdf_brute": (None, [_P, _P, _I64, _P, _P, _P, _P, _I64, _P, _P]),
            "port_mesh_sdf_flat": (None, [_P, _P, _I64, _P, _P, _P, _P, _I64, _P, _P]),
            "port_dcel_face_sd": (_D, [_P, _P, _P, _P, _P]),
            "port_knn_brute": (None, [_P, _I64, _P, _I64, C.c_int, _P, _P]),
            "port_knn_brute_self": (None, [_P, _I64, C.c_int, _P, _P]),
            "port_sphere_sd": (_D, [_P, _D, _P]),
            "port_rotate_point": (None, [_D, C.c_int, _P, _P]),
            "port_scene_brute": (None, [_I64, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _P]),
        }
        for k, (r, a) in sig.items():
            fn = getattr(lib, k)
            fn.restype = r
            fn.argtypes = a
        self.lib = lib

    def triangle_sd(self, v, fn, vn, en, p, scalar=False) -> float:
        a = [np.ascontiguousarray(x, np.float64).ravel() for x in (v, fn, vn, en, p)]
        f = self.lib.port_triangle_sd_scalar if scalar else self.lib.port_triangle_sd
        return float(f(*[_ptr(x) for x in a]))

    def mesh_normals(self, v, f):
        v = np.ascontiguousarray(v, np.float64)
        f = np.ascontiguousarray(f, np.int64)
        t = f.shape[0]
        tn, vn, en = np.empty((t, 3)), np.empty((v.shape[0], 3)), np.empty((t, 3, 3))
        rc = self.lib.port_mesh_normals(_ptr(v), v.shape[0], _ptr(f), t, _ptr(tn), _ptr(vn), _ptr(en))
        assert rc == 0
        return tn, vn[f], en  # corner vertex normals (T,3,3)

    def mesh_sdf_brute(self, v, f, p, normals=None):
        v = np.ascontiguousarray(v, np.float64)
        f64 = np.ascontiguousarray(f, np.int64)
        if normals is None:
            tn, vn, en = self.mesh_normals(v, f64)
            vn_v = np.empty((v.shape[0], 3))
            vn_v[f64.ravel()] = vn.reshape(-1, 3)
        else:
            tn, vn_v, en = normals
        tn, vn_v, en = (np.ascontiguousarray(x, np.float64) for x in (tn, vn_v, en))
        p = np.ascontiguousarray(p, np.float64).reshape(-1, 3)
        out = np.empty(p.shape[0])
        tri = np.empty(p.shape[0], np.int64)
        self.lib.port_mesh_sdf_brute(_ptr(v), _ptr(f64), f64.shape[0], _ptr(tn), _ptr(vn_v), _ptr(en), _ptr(p),
                                     p.shape[0], _ptr(out), _ptr(tri))
        return out, tri

    def mesh_sdf_flat(self, v, f, p):
        """FlatMeshSDF (DCEL faces, Direct2 search): values and winning faces."""
        v = np.ascontiguousarray(v, np.float64)
        f64 = np.ascontiguousarray(f, np.int64)
        tn, vn, en = self.mesh_normals(v, f64)
        vn_v = np.empty((v.shape[0], 3))
        vn_v[f64.ravel()] = vn.reshape(-1, 3)
        tn, vn_v, en = (np.ascontiguousarray(x, np.float64) for x in (tn, vn_v, en))
        p = np.ascontiguousarray(p, np.float64).reshape(-1, 3)
        out = np.empty(p.shape[0])
        tri = np.empty(p.shape[0], np.int64)
        self.lib.port_mesh_sdf_flat(_ptr(v), _ptr(f64), f64.shape[0], _ptr(tn), _ptr(vn_v), _ptr(en), _ptr(p),
                                    p.shape[0], _ptr(out), _ptr(tri))
        return out, tri

    def dcel_face_sd(self, v, fn, vn, en, p):
        """One triangle as a DCEL face: v (3,3) loop order, fn the DCEL face normal, vn (3,3), en (3,3)."""
        a = [np.ascontiguousarray(x, np.float64) for x in (v, fn, vn, en, p)]
        return float(self.lib.port_dcel_face_sd(*[_ptr(x) for x in a]))

    def knn_brute(self, pts, q, k):
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        q = np.ascontiguousarray(q, np.float32).reshape(-1, 3)
        idx = np.empty((q.shape[0], k), np.int32)
        d2 = np.empty((q.shape[0], k), np.float32)
        self.lib.port_knn_brute(_ptr(pts), pts.shape[0], _ptr(q), q.shape[0], k, _ptr(idx), _ptr(d2))
        return idx, d2

    def knn_brute_self(self, pts, k):
        """Every point's k nearest other points, lexicographic (d2, index)."""
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        idx = np.empty((pts.shape[0], k), np.int32)
        d2 = np.empty((pts.shape[0], k), np.float32)
        self.lib.port_knn_brute_self(_ptr(pts), pts.shape[0], k, _ptr(idx), _ptr(d2))
        return idx, d2

    def scene_brute(self, spheres, meshes, poses, p):
        spheres = np.ascontiguousarray(spheres, np.float64).reshape(-1, 4)
        vs, fs, tns, vns, ens = [], [], [], [], []
        for v, f in meshes:
            v = np.asarray(v, np.float64)
            f = np.asarray(f, np.int64)
            tn, vn, en = self.mesh_normals(v, f)
            vn_v = np.empty((v.shape[0], 3))
            vn_v[f.ravel()] = vn.reshape(-1, 3)
            vs.append(v), fs.append(f), tns.append(tn), vns.append(vn_v), ens.append(en)
        cat = lambda xs, shp: np.ascontiguousarray(np.concatenate(xs) if xs else np.zeros(shp))
        V, F = cat(vs, (0, 3)), cat(fs, (0, 3)).astype(np.int64)
        TN, VN, EN = cat(tns, (0, 3)), cat(vns, (0, 3)), cat(ens, (0, 3, 3))
        vcnt = np.array([v.shape[0] for v in vs], np.int64)
        fcnt = np.array([f.shape[0] for f in fs], np.int64)
        voff = np.ascontiguousarray(np.concatenate([[0], np.cumsum(vcnt)[:-1]]).astype(np.int64))
        foff = np.ascontiguousarray(np.concatenate([[0], np.cumsum(fcnt)[:-1]]).astype(np.int64))
        poses = np.ascontiguousarray(poses, np.float64).reshape(-1, 5)
        p = np.ascontiguousarray(p, np.float64).reshape(-1, 3)
        out = np.empty(p.shape[0])
        self.lib.port_scene_brute(spheres.shape[0], _ptr(spheres), len(meshes), _ptr(V), _ptr(voff), _ptr(foff),
                                  _ptr(fcnt), _ptr(F), _ptr(TN), _ptr(VN), _ptr(EN), _ptr(poses), _ptr(p),
                                  p.shape[0], _ptr(out))
        return out


_ref_cache = None
_port_cache = None


def ref_available() -> bool:
    return os.path.exists(ref_lib_path())


_ref_timing_cache = None


def ref(timing: bool = False) -> _Ref:
    """The reference oracle: the parity build, or with ``timing`` the build bench.py times (see
    ref_lib_path); both are the unmodified reference behind the same extern "C" harness."""
    global _ref_cache, _ref_timing_cache
    cached = _ref_timing_cache if timing else _ref_cache
    if cached is None:
        path = ref_lib_path(timing)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference sources exist")
        cached = _Ref(path)
        if timing:
            _ref_timing_cache = cached
        else:
            _ref_cache = cached
    return cached


def port() -> _Port:
    global _port_cache
    if _port_cache is None:
        if not os.path.exists(PORT_LIB):
            build()
        _port_cache = _Port(PORT_LIB)
    return _port_cache
