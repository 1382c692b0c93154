"""ctypes binding of the C ABI declared in include/r2.h.

The native library is required: importing this module raises if
``_lib/librenderer2.so`` is missing (there is no Python or CPU fallback for
the hot paths).  The library itself is opened on the first use of ``lib``,
so that modules which only describe inputs (structures, seeded generators)
can be imported by code that must not load it, such as the CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "librenderer2.so")


class R2Error(RuntimeError):
    def __init__(self, status: int, name: str, message: str):
        super().__init__(f"{name}: {message}")
        self.status = status
        self.name = name


class Voxel(C.Structure):
    _fields_ = [("density", C.c_float), ("sigma", C.c_uint16 * 3), ("r", C.c_uint16 * 3),
                ("diffuse", C.c_uint8 * 3), ("specular", C.c_uint8 * 3), ("normal", C.c_uint16 * 3),
                ("ior", C.c_uint16), ("pad", C.c_uint16)]


VOXEL_DTYPE = np.dtype([("density", "<f4"), ("sigma", "<u2", 3), ("r", "<u2", 3), ("diffuse", "u1", 3),
                        ("specular", "u1", 3), ("normal", "<u2", 3), ("ior", "<u2"), ("pad", "<u2")])
assert VOXEL_DTYPE.itemsize == 32


class Material(C.Structure):
    _fields_ = [("diffuse", C.c_float * 3), ("specular", C.c_float * 3), ("alpha_x", C.c_float),
                ("alpha_y", C.c_float), ("eta_i", C.c_float), ("eta_t", C.c_float),
                ("diffuse_roughness", C.c_float), ("pad", C.c_float)]


class MaterialMaps(C.Structure):
    _fields_ = [("albedo", C.c_char_p), ("specular", C.c_char_p), ("normal", C.c_char_p), ("alpha", C.c_char_p)]


class FilterParams(C.Structure):
    _fields_ = [("min_voxel_size", C.c_float), ("lods", C.c_uint32), ("samples_per_voxel", C.c_uint32),
                ("sigma_t", C.c_float), ("estimation_iterations", C.c_uint32), ("alpha", C.c_float),
                ("clip_rays", C.c_uint32), ("seed", C.c_uint32), ("sggx_projection", C.c_uint32),
                ("sggx_floor", C.c_float)]


class FilterGrid(C.Structure):
    _fields_ = [("num_voxels", C.c_int32 * 3), ("index_to_model", C.c_float * 12),
                ("model_to_index", C.c_float * 12), ("model_to_world", C.c_float * 12),
                ("world_to_model", C.c_float * 12), ("world_bb_min", C.c_float * 3),
                ("world_bb_max", C.c_float * 3), ("voxel_size", C.c_float)]


# r2_lod_camera and r2_lod_volume (screen-space LOD selection)
LOD_CAMERA_DTYPE = np.dtype([("world_to_view", "<f8", 16), ("pos", "<f8", 3), ("near_plane_distance", "<f8"),
                             ("pixel_size", "<f8"), ("pixel_area", "<f8"), ("sensor_width", "<f8"),
                             ("sensor_height", "<f8"), ("far_scale", "<f8")])
LOD_VOLUME_DTYPE = np.dtype([("voxel_size", "<f8"), ("bb_min", "<f8", 3), ("bb_max", "<f8", 3),
                             ("num_voxels", "<f8", 3), ("corners", "<f8", (8, 3))])
assert LOD_CAMERA_DTYPE.itemsize == 200 and LOD_VOLUME_DTYPE.itemsize == 272


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"native library missing: {LIB_PATH} (run __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    P = C.c_void_p
    u32, i32, f32, sz = C.c_uint32, C.c_int32, C.c_float, C.c_size_t
    sigs = {
        "r2_status_string": (C.c_char_p, [C.c_int]),
        "r2_last_error": (C.c_char_p, []),
        "r2_version": (C.c_int, []),
        "r2_set_bvh_method": (C.c_int, [C.c_int]),
        "r2_get_bvh_method": (C.c_int, []),
        "r2_scene_bvh_info": (C.c_int, [P, P, P, P]),
        "r2_scene_add_mesh_asset": (C.c_int, [P, P, C.c_uint32, P, C.c_uint32, P, P, P, P, P]),
        "r2_scene_add_mesh_instance": (C.c_int, [P, C.c_uint32, P, C.c_uint32]),
        "r2_filter_setup_grid": (C.c_int, [P, P, P, f32, P]),
        "r2_filter_mesh": (C.c_int, [P, u32, P, u32, P, P, P, P, f32, P, P, P, sz]),
        "r2_filter_scene_create": (C.c_int, [P, u32, P, u32, P, P, P, P]),
        "r2_filter_scene_destroy": (C.c_int, [P]),
        "r2_filter_scene_create_textured": (C.c_int, [P, u32, P, u32, P, P, P, P, P, P]),
        "r2_filter_scene_grid": (C.c_int, [P, f32, P]),
        "r2_filter_scene_run": (C.c_int, [P, P, P, P, P, P, P, P]),
        "r2_filter_scene_run_eig": (C.c_int, [P, P, P, P, P, P, P, P, P]),
        "r2_filter_scene_count": (C.c_int, [P, P, P, P, P]),
        "r2_filter_scene_bvh": (C.c_int, [P, P, sz, P, sz, P, P]),
        "r2_scene_create": (C.c_int, [P]),
        "r2_scene_destroy": (C.c_int, [P]),
        "r2_scene_add_mesh": (C.c_int, [P, P, u32, P, u32, P, P, P, u32]),
        "r2_scene_add_mesh_textured": (C.c_int, [P, P, u32, P, u32, P, P, P, P, P, u32]),
        "r2_scene_add_shape": (C.c_int, [P, C.c_int, P, f32, P, P, u32]),
        "r2_scene_set_envmap": (C.c_int, [P, P, u32, u32]),
        "r2_scene_add_medium": (C.c_int, [P, C.c_char_p, P, P, P, P, P, u32]),
        "r2_scene_add_medium_hg": (C.c_int, [P, C.c_char_p, P, P, f32, P, P, P, u32]),
        "r2_filter_run_mesh": (C.c_int, [P, u32, P, u32, P, P, P, P, P, P, C.c_char_p, C.c_char_p, P]),
        "r2_scene_commit": (C.c_int, [P]),
        "r2_scene_rebuild": (C.c_int, [P, P]),
        "r2_scene_set_vertices": (C.c_int, [P, P, P, u32, P]),
        "r2_render_device": (C.c_int, [P, P, P, P, P, P]),
        "r2_render_host": (C.c_int, [P, P, P, P]),
        "r2_scene_set_tuning": (C.c_int, [P, P]),
        "r2_scene_get_tuning": (C.c_int, [P, P]),
        "r2_scene_autotune": (C.c_int, [P, P, P, P]),
        "r2_scene_wave_samples": (C.c_int, [P, P, P, P]),
        "r2_render_batch_create": (C.c_int, [P, P, P, P, u32, P]),
        "r2_render_batch_destroy": (C.c_int, [P]),
        "r2_render_batch_run": (C.c_int, [P, P, P]),
        "r2_server_create": (C.c_int, [u32, C.c_uint64, P]),
        "r2_server_destroy": (C.c_int, [P]),
        "r2_server_submit_render": (C.c_int, [P, P, P, P, P, P]),
        "r2_server_render_bytes": (C.c_int, [P, P, P, P]),
        "r2_server_submit_filter": (C.c_int, [P, P, P, P, u32, P, P]),
        "r2_server_wait": (C.c_int, [P, C.c_uint64, C.c_double, P]),
        "r2_server_stats": (C.c_int, [P, P]),
        "r2_config_load": (C.c_int, [C.c_char_p, P]),
        "r2_config_free": (C.c_int, [P]),
        "r2_config_info_get": (C.c_int, [P, P]),
        "r2_filter_run": (C.c_int, [P, C.c_char_p, P]),
        "r2_render": (C.c_int, [P, P, P, P]),
        "r2_tonemap": (C.c_int, [P, u32, u32, f32, P, P]),
        "r2_write_png": (C.c_int, [C.c_char_p, P, u32, u32, C.c_int]),
        "r2_write_jpg": (C.c_int, [C.c_char_p, P, u32, u32, C.c_int, C.c_int]),
        "r2_read_png": (C.c_int, [C.c_char_p, P, sz, P, P, P]),
        "r2_read_hdr": (C.c_int, [C.c_char_p, P, sz, P, P]),
        "r2_write_hdr": (C.c_int, [C.c_char_p, P, u32, u32]),
        "r2_obj_info": (C.c_int, [C.c_char_p, C.c_char_p, P, P, P, P]),
        "r2_select_lods": (C.c_int, [P, P, P, P, u32, P, P, P, u32, C.c_double, C.c_double, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


if not os.path.exists(LIB_PATH):
    raise ImportError(f"native library missing: {LIB_PATH} (run __graft_entry__.build())")


def __getattr__(name):
    if name == "lib":
        loaded = _load()
        globals()["lib"] = loaded
        return loaded
    raise AttributeError(name)


def check(status: int) -> None:
    if status != 0:
        name = lib.r2_status_string(status).decode()
        msg = lib.r2_last_error().decode()
        raise R2Error(status, name, msg)


def ptr(a):
    """Host pointer of a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


def identity43() -> np.ndarray:
    m = np.zeros(12, np.float32)
    m[0] = m[4] = m[8] = 1.0
    return m
