"""ctypes binding of the C ABI declared in include/ebgeometry_b200.h.

The shared library ``libebgb200.so`` is built in-tree (``ebgeometry_b200/csrc/Makefile``).  There
is no CPU fallback: if the library cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libebgb200.so")


class BuildOpts(C.Structure):
    _fields_ = [("build", C.c_int32), ("leaf_size", C.c_int32), ("device", C.c_int32),
                ("flags", C.c_int32)]


class PhaseTimings(C.Structure):
    _fields_ = [("order_ms", C.c_float), ("traverse_ms", C.c_float), ("band_ms", C.c_float),
                ("total_ms", C.c_float)]


class QueryOpts(C.Structure):
    _fields_ = [("band", C.c_double), ("no_sort", C.c_int32), ("no_fp64_band", C.c_int32),
                ("seed", C.c_void_p), ("warps_per_block", C.c_int32), ("occupancy", C.c_int32),
                ("timings", C.POINTER(PhaseTimings)), ("radius_hint", C.c_void_p), ("queue_chunk", C.c_int32),
                ("top_nodes", C.c_int32), ("node_width", C.c_int32)]


class SeedOpts(C.Structure):
    _fields_ = [("num_samples", C.c_int64), ("steps", C.c_int32), ("batch", C.c_int32),
                ("log2_table", C.c_int32), ("base_resolution", C.c_int32), ("max_resolution", C.c_int32),
                ("learning_rate", C.c_float), ("surface_band", C.c_float), ("coverage", C.c_float),
                ("rng_seed", C.c_uint64), ("lo", C.c_double * 3), ("hi", C.c_double * 3)]


class SeedReport(C.Structure):
    _fields_ = [("train_seconds", C.c_float), ("final_loss", C.c_float), ("alpha", C.c_float),
                ("beta", C.c_float), ("coverage", C.c_float), ("mean_abs_err", C.c_float),
                ("far_tau", C.c_float), ("max_abs_err_far", C.c_float),
                ("validation_samples", C.c_int64), ("train_samples", C.c_int64)]


class MeshInfo(C.Structure):
    _fields_ = [("num_triangles", C.c_int64), ("num_vertices", C.c_int64),
                ("num_nodes", C.c_int64), ("num_leaves", C.c_int64), ("depth", C.c_int32),
                ("leaf_size", C.c_int32), ("lo", C.c_double * 3), ("hi", C.c_double * 3),
                ("diagonal", C.c_double), ("device_bytes", C.c_int64)]


class QueryStats(C.Structure):
    _fields_ = [("nodes_visited", C.c_int64), ("leaves_visited", C.c_int64),
                ("triangles_tested", C.c_int64), ("band_queries", C.c_int64),
                ("seed_fallbacks", C.c_int64), ("packets", C.c_int64), ("packet_pops", C.c_int64),
                ("packet_nodes", C.c_int64), ("packet_leaves", C.c_int64), ("packet_triangles", C.c_int64),
                ("boxes_tested", C.c_int64), ("packet_boxes", C.c_int64), ("cut_packets", C.c_int64),
                ("cut_entries", C.c_int64), ("packet_triangle_records", C.c_int64)]


class AttachOpts(C.Structure):
    _fields_ = [("cells_per_axis", C.c_int32), ("max_entries", C.c_int32), ("margin_cells", C.c_float),
                ("radius_mode", C.c_int32), ("no_anchors", C.c_int32)]


class AttachReport(C.Structure):
    _fields_ = [("cells_per_axis", C.c_int32), ("max_entries", C.c_int32), ("cells", C.c_int64),
                ("cut_entries", C.c_int64), ("empty_cells", C.c_int64), ("device_bytes", C.c_int64),
                ("build_ms", C.c_float), ("mean_radius", C.c_float)]


EBG_OK = 0
STATUS_NAMES = {0: "EBG_OK", 1: "EBG_ERR_INVALID", 2: "EBG_ERR_CUDA", 3: "EBG_ERR_NO_MEMORY",
                4: "EBG_ERR_TRAVERSAL", 5: "EBG_ERR_NOT_FOUND", 6: "EBG_ERR_TOO_LARGE"}

_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32
_D = C.c_double

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "ebg_last_error": (C.c_char_p, []),
    "ebg_version": (C.c_char_p, []),
    "ebg_device_count": (C.c_int, []),
    "ebg_sample_points": (C.c_int, [_I64, C.c_uint64, _P]),
    "ebg_mesh_create": (C.c_int, [_P, _I64, _P, _I64, C.POINTER(BuildOpts), C.POINTER(_P)]),
    "ebg_mesh_create_with_normals": (C.c_int, [_P, _I64, _P, _I64, _P, _P, C.POINTER(BuildOpts),
                                               C.POINTER(_P)]),
    "ebg_compute_pseudonormals": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _P]),
    "ebg_mesh_destroy": (C.c_int, [_P]),
    "ebg_mesh_refit": (C.c_int, [_P, _P, _I64, _P]),
    "ebg_mesh_refit_device": (C.c_int, [_P, _P, _I64, _P]),
    "ebg_mesh_get_info": (C.c_int, [_P, C.POINTER(MeshInfo)]),
    "ebg_mesh_get_normals": (C.c_int, [_P, _P, _P, _P]),
    "ebg_mesh_signed_distance": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_soup_read": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "ebg_soup_sizes": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(_I64)]),
    "ebg_soup_copy": (C.c_int, [_P, _P, _P]),
    "ebg_soup_destroy": (C.c_int, [_P]),
    "ebg_soup_num_corners": (C.c_int, [_P, C.POINTER(_I64)]),
    "ebg_soup_copy_polygons": (C.c_int, [_P, _P, _P, _P]),
    "ebg_polymesh_create": (C.c_int, [_P, _I64, _P, _P, _I64, C.POINTER(BuildOpts), C.POINTER(_P)]),
    "ebg_polymesh_create_from_file": (C.c_int, [C.c_char_p, C.POINTER(BuildOpts), C.POINTER(_P)]),
    "ebg_polymesh_destroy": (C.c_int, [_P]),
    "ebg_compute_polygon_normals": (C.c_int, [_P, _I64, _P, _P, _I64, _P, _P, _P, _P]),
    "ebg_polymesh_get_info": (C.c_int, [_P, C.POINTER(MeshInfo), C.POINTER(_I64)]),
    "ebg_polymesh_get_normals": (C.c_int, [_P, _P, _P, _P, _P]),
    "ebg_polymesh_signed_distance": (C.c_int, [_P, _P, _I64, _P, _P, _P]),
    "ebg_polymesh_signed_distance_host": (C.c_int, [_P, _P, _I64, _P, _P, _P]),
    "ebg_polymesh_signed_distance_flat": (C.c_int, [_P, _P, _I64, _P, _P, _P]),
    "ebg_polymesh_signed_distance_flat_host": (C.c_int, [_P, _P, _I64, _P, _P, _P]),
    "ebg_polymesh_check_status": (C.c_int, [_P, _P]),
    "ebg_mesh_create_from_file": (C.c_int, [C.c_char_p, C.POINTER(BuildOpts), C.POINTER(_P)]),
    "ebg_mesh_signed_distance_host": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_mesh_signed_distance_noalloc": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_mesh_signed_distance_f64": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_mesh_signed_distance_f64_host": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_mesh_signed_distance_dcel_f64": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_mesh_signed_distance_dcel_f64_host": (C.c_int, [_P, _P, _I64, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_mesh_signed_distance_flat_f64": (C.c_int, [_P, _P, _I64, _P, _P, _P]),
    "ebg_mesh_signed_distance_flat_f64_host": (C.c_int, [_P, _P, _I64, _P, _P, _P]),
    "ebg_mesh_signed_distance_stats": (C.c_int, [_P, _P, _I64, _P, C.POINTER(QueryOpts),
                                                 C.POINTER(QueryStats), _P]),
    "ebg_mesh_value": (C.c_int, [_P, _D, _D, _D, C.POINTER(_D)]),
    "ebg_mesh_autotune": (C.c_int, [_P, _P, _I64, _P, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_I32),
                                    C.POINTER(_I32), C.POINTER(C.c_float), _P]),
    "ebg_mesh_widen": (C.c_int, [_P, C.POINTER(_I64), C.POINTER(_I32)]),
    "ebg_check_status": (C.c_int, [_P, _P]),
    "ebg_cloud_create": (C.c_int, [_P, _I64, C.POINTER(BuildOpts), C.POINTER(_P)]),
    "ebg_cloud_create_device": (C.c_int, [_P, _I64, C.POINTER(BuildOpts), C.POINTER(_P), _P]),
    "ebg_cloud_destroy": (C.c_int, [_P]),
    "ebg_cloud_size": (_I64, [_P]),
    "ebg_cloud_tree_info": (C.c_int, [_P, _P, _P, _P]),
    "ebg_cloud_knn": (C.c_int, [_P, _P, _I64, _I32, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_cloud_knn_host": (C.c_int, [_P, _P, _I64, _I32, _P, _P, C.POINTER(QueryOpts), _P]),
    "ebg_cloud_self_knn": (C.c_int, [_P, _I32, _P, _P, _P]),
    "ebg_cloud_self_knn_points": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _P]),
    "ebg_cloud_self_knn_host": (C.c_int, [_P, _I32, _P, _P, _P]),
    "ebg_cloud_self_knn_points_host": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _P]),
    "ebg_cloud_check_status": (C.c_int, [_P, _P]),
    "ebg_grid_create": (C.c_int, [_P, _I64, C.c_double, _I32, C.POINTER(_P)]),
    "ebg_grid_destroy": (C.c_int, [_P]),
    "ebg_grid_size": (_I64, [_P]),
    "ebg_grid_info": (C.c_int, [_P, _P, _P]),
    "ebg_grid_knn": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _P]),
    "ebg_grid_knn_host": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _P]),
    "ebg_grid_self_knn": (C.c_int, [_P, _I32, _P, _P, _P]),
    "ebg_grid_self_knn_host": (C.c_int, [_P, _I32, _P, _P, _P]),
    "ebg_grid_self_knn_points": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _P]),
    "ebg_grid_self_knn_points_host": (C.c_int, [_P, _P, _I64, _I32, _P, _P, _P]),
    "ebg_grid_check_status": (C.c_int, [_P, _P]),
    "ebg_scene_create": (C.c_int, [_I64, _P, _I64, _P, _P, C.POINTER(BuildOpts), C.POINTER(_P)]),
    "ebg_scene_destroy": (C.c_int, [_P]),
    "ebg_scene_num_objects": (_I64, [_P]),
    "ebg_scene_value": (C.c_int, [_P, _P, _I64, _P, C.POINTER(QueryOpts), _P]),
    "ebg_scene_value_host": (C.c_int, [_P, _P, _I64, _P, C.POINTER(QueryOpts), _P]),
    "ebg_scene_check_status": (C.c_int, [_P, _P]),
    "ebg_scene_eval_batches": (C.c_int, [_P, _P, _I32, _I64, C.POINTER(QueryOpts), _P]),
    "ebg_scene_autotune": (C.c_int, [_P, _P, _I64, C.POINTER(_I32), C.POINTER(C.c_float), _P]),
    "ebg_seed_create": (C.c_int, [C.POINTER(SeedOpts), C.POINTER(_P)]),
    "ebg_seed_train": (C.c_int, [_P, C.POINTER(SeedOpts), C.POINTER(_P), C.POINTER(SeedReport), _P]),
    "ebg_seed_destroy": (C.c_int, [_P]),
    "ebg_seed_get_report": (C.c_int, [_P, C.POINTER(SeedReport)]),
    "ebg_seed_predict": (C.c_int, [_P, _P, _I64, _P, _P]),
    "ebg_seed_save": (C.c_int, [_P, C.c_char_p]),
    "ebg_seed_load": (C.c_int, [C.c_char_p, _I32, C.POINTER(_P)]),
    "ebg_seed_get_params": (C.c_int, [_P, _P, _P]),
    "ebg_seed_set_params": (C.c_int, [_P, _P, _P]),
    "ebg_seed_gradients": (C.c_int, [_P, _P, _P, _I32, C.c_float, C.POINTER(C.c_float), _P, _P]),
    "ebg_seed_attach": (C.c_int, [_P, _P, C.POINTER(AttachOpts), C.POINTER(AttachReport), _P]),
    "ebg_seed_detach": (C.c_int, [_P]),
}


class EbgError(RuntimeError):
    """A C ABI call returned a non-zero ebg_status."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C ebgeometry_b200/csrc` (or "
            "__graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int) -> None:
    if status != EBG_OK:
        raise EbgError(status, lib.ebg_last_error().decode())
