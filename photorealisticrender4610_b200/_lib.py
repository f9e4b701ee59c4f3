"""ctypes binding to libprr.so (the C ABI declared in include/prr.h).

The library is built in-tree (``photorealisticrender4610_b200/build.py``).
Loading fails loudly when it is missing: there is no CPU fallback. With
PRR_LIBRARY=checked in the environment the checked build (libprr_checked.so,
device-side bounds tests reported by prr_check_status) is loaded instead.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / ("libprr_checked.so" if os.environ.get("PRR_LIBRARY") == "checked"
                  else "libprr.so")
HEADER_DIR = PKG.parent / "include"

PRR_OK = 0
ERRORS = {
    -1: "PRR_ERR_INVALID_ARGUMENT", -2: "PRR_ERR_CUDA", -3: "PRR_ERR_OUT_OF_MEMORY",
    -4: "PRR_ERR_NOT_BUILT", -5: "PRR_ERR_UNSUPPORTED", -6: "PRR_ERR_TIMEOUT",
    -7: "PRR_ERR_BUDGET", -8: "PRR_ERR_INTERNAL",
}


class PrrError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class prr_camera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3),
                ("fovv", C.c_float), ("fovh", C.c_float), ("aperture", C.c_float),
                ("focus_distance", C.c_float)]


class prr_trace_config(C.Structure):
    _fields_ = [("block_size", C.c_int), ("persistent", C.c_int), ("blocks_per_sm", C.c_int),
                ("batch", C.c_int), ("leaf_batch", C.c_int), ("sort_rays", C.c_int)]


class prr_wavefront_config(C.Structure):
    _fields_ = [("paths_per_pass", C.c_int64), ("block_size", C.c_int), ("use_graphs", C.c_int),
                ("stack_smem", C.c_int), ("ordered", C.c_int), ("refill", C.c_int)]


class prr_medium(C.Structure):
    _fields_ = [("sigma_a", C.c_float), ("sigma_s", C.c_float), ("sigma_t", C.c_float),
                ("g", C.c_float), ("bounded", C.c_int), ("bounds_min", C.c_float * 3),
                ("bounds_max", C.c_float * 3)]


class prr_server_config(C.Structure):
    _fields_ = [("device_budget_bytes", C.c_int64), ("max_active", C.c_int),
                ("samples_per_step", C.c_int64), ("fail_every_nth_admission", C.c_int),
                ("integrator", C.c_int), ("paths_per_launch", C.c_int64)]


class prr_request_info(C.Structure):
    _fields_ = [("status", C.c_int), ("error", C.c_int), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double), ("samples", C.c_int64),
                ("rays", C.c_uint64)]


class prr_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("active", C.c_int64), ("queued", C.c_int64), ("samples", C.c_int64),
                ("rays", C.c_uint64), ("steps", C.c_int64), ("busy_s", C.c_double),
                ("admit_s", C.c_double), ("complete_s", C.c_double),
                ("bytes_in_use", C.c_int64), ("now_s", C.c_double), ("launches", C.c_int64)]


class prr_scene_stats(C.Structure):
    _fields_ = [("n_objects", C.c_int64), ("n_triangles", C.c_int64), ("n_nodes", C.c_int64),
                ("tlas_depth", C.c_int32), ("blas_depth", C.c_int32),
                ("device_bytes", C.c_int64), ("total_emit_area", C.c_float),
                ("last_render_launches", C.c_int64)]


class prr_render_count(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "closest_rays", "closest_nodes", "closest_tris", "closest_objects",
        "shadow_rays", "shadow_nodes", "shadow_tris", "shadow_objects",
        "misses", "delta_hits", "surface_hits")]


class prr_render_settings(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("min_spp", C.c_int),
                ("max_spp", C.c_int), ("max_depth", C.c_int), ("variance_threshold", C.c_float),
                ("indirect_clamp", C.c_float), ("mode", C.c_int), ("seed", C.c_uint64),
                ("x0", C.c_int), ("y0", C.c_int), ("x1", C.c_int), ("y1", C.c_int),
                ("sample_offset", C.c_int), ("slices", C.c_int)]


class prr_request(C.Structure):
    _fields_ = [("scene", C.c_int), ("settings", prr_render_settings), ("out_rgb", C.c_void_p)]


_vp = C.c_void_p
_SIGS = {
    "prr_abi_version": (C.c_int, []),
    "prr_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "prr_bvh_build": (C.c_int64, [_vp, _vp, C.c_int64, C.c_int, _vp, _vp, _vp, _vp, _vp,
                                  C.POINTER(C.c_int32)]),
    "prr_scene_create": (C.c_int, [C.POINTER(_vp)]),
    "prr_scene_destroy": (C.c_int, [_vp]),
    "prr_scene_add_material": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "prr_scene_add_mesh": (C.c_int, [_vp, _vp, C.c_int64, C.c_int, C.POINTER(C.c_int)]),
    "prr_scene_add_mesh_attr": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, C.c_int,
                                          C.POINTER(C.c_int)]),
    "prr_scene_add_texture": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(C.c_int)]),
    "prr_scene_set_material_textures": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int,
                                                  C.c_int]),
    "prr_write_image": (C.c_int, [C.c_char_p, _vp, C.c_int, C.c_int]),
    "prr_sample_count_image": (C.c_int, [_vp, C.c_int64, C.c_int, _vp]),
    "prr_scene_add_gltf": (C.c_int, [_vp, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "prr_scene_add_obj": (C.c_int, [_vp, C.c_char_p, _vp, C.c_int, C.POINTER(C.c_int)]),
    "prr_obj_read": (C.c_int, [C.c_char_p, _vp, _vp, C.c_int64, C.POINTER(C.c_int64)]),
    "prr_scene_export_mesh": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                        _vp, _vp, _vp, _vp]),
    "prr_scene_export_material": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), _vp, _vp]),
    "prr_scene_export_texture": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                           C.POINTER(C.c_int), _vp]),
    "prr_scene_add_sphere": (C.c_int, [_vp, C.POINTER(C.c_float), C.c_float, C.c_int,
                                       C.POINTER(C.c_int)]),
    "prr_scene_set_background": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "prr_scene_set_env": (C.c_int, [_vp, _vp, C.c_int, C.c_int]),
    "prr_scene_set_camera": (C.c_int, [_vp, C.POINTER(prr_camera), C.c_int, C.c_int]),
    "prr_scene_build": (C.c_int, [_vp, _vp]),
    "prr_scene_stats_get": (C.c_int, [_vp, C.POINTER(prr_scene_stats)]),
    "prr_scene_export_nodes": (C.c_int64, [_vp, C.c_int, _vp, _vp, _vp, _vp, _vp]),
    "prr_mesh_intersect": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int64, _vp, _vp, _vp,
                                     C.POINTER(prr_trace_config), _vp]),
    "prr_mesh_intersect_host": (C.c_int, [_vp, C.c_int, _vp, _vp, C.c_int64, _vp, _vp, _vp,
                                          _vp]),
    "prr_mesh_occluded": (C.c_int, [_vp, C.c_int, _vp, _vp, _vp, C.c_int64, _vp, _vp]),
    "prr_scene_intersect": (C.c_int, [_vp, _vp, _vp, C.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "prr_scene_occluded": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, _vp, _vp]),
    "prr_render": (C.c_int, [_vp, C.POINTER(prr_render_settings), _vp, _vp, _vp, _vp]),
    "prr_render_counts": (C.c_int, [_vp, C.POINTER(prr_render_settings), _vp,
                                    C.POINTER(prr_render_count), _vp]),
    "prr_check_status": (C.c_int, [_vp, _vp, C.c_int]),
    "prr_photon_map_create": (C.c_int, [C.POINTER(_vp)]),
    "prr_photon_map_destroy": (C.c_int, [_vp]),
    "prr_photon_emit": (C.c_int, [_vp, _vp, C.c_int64, C.c_uint64, C.c_int, _vp]),
    "prr_photon_set": (C.c_int, [_vp, _vp, C.c_int64, _vp]),
    "prr_photon_build": (C.c_int, [_vp, C.c_float, _vp]),
    "prr_photon_info": (C.c_int, [_vp, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "prr_photon_launches": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "prr_photon_export": (C.c_int, [_vp, _vp, _vp, _vp]),
    "prr_photon_gather": (C.c_int, [_vp, _vp, C.c_int64, C.c_int, _vp, _vp]),
    "prr_render_caustics": (C.c_int, [_vp, _vp, C.POINTER(prr_render_settings), C.c_int, _vp,
                                      _vp]),
    "prr_render_caustics_counts": (C.c_int, [_vp, _vp, C.POINTER(prr_render_settings), C.c_int,
                                             _vp, _vp, _vp]),
    "prr_medium_preset": (C.c_int, [C.c_int, C.POINTER(prr_medium)]),
    "prr_medium_intersect": (C.c_int, [C.POINTER(prr_medium), _vp, _vp, C.c_int64, _vp, _vp,
                                       _vp, _vp]),
    "prr_phase_hg": (C.c_int, [_vp, C.c_int64, C.c_float, _vp, _vp]),
    "prr_phase_hg_sample": (C.c_int, [_vp, C.c_int64, C.c_float, C.c_uint64, _vp, _vp]),
    "prr_server_create": (C.c_int, [C.POINTER(prr_server_config), C.POINTER(_vp)]),
    "prr_server_destroy": (C.c_int, [_vp]),
    "prr_server_add_scene": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
    "prr_server_submit": (C.c_int, [_vp, _vp, C.POINTER(C.c_uint64)]),
    "prr_server_cancel": (C.c_int, [_vp, C.c_uint64]),
    "prr_server_poll": (C.c_int, [_vp, C.c_uint64, C.POINTER(prr_request_info)]),
    "prr_server_wait": (C.c_int, [_vp, C.c_uint64, C.c_double, C.POINTER(prr_request_info)]),
    "prr_server_stats_get": (C.c_int, [_vp, C.POINTER(prr_server_stats)]),
    "prr_tonemap": (C.c_int, [C.c_int, C.c_float, _vp, C.c_int64, _vp, _vp, _vp]),
    "prr_render_noalloc": (C.c_int, [_vp, C.POINTER(prr_render_settings), _vp, _vp, _vp]),
    "prr_scene_set_wavefront": (C.c_int, [_vp, C.POINTER(prr_wavefront_config)]),
    "prr_autotune": (C.c_int, [_vp, C.POINTER(prr_render_settings),
                               C.POINTER(prr_wavefront_config), _vp]),
    "prr_cast_samples": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int64, C.c_uint64, C.c_int, C.c_float,
                                   _vp, _vp]),
    "prr_cast_rays": (C.c_int, [_vp, _vp, _vp, C.c_int64, C.c_uint64, C.c_int, C.c_float, _vp,
                                _vp]),
    "prr_camera_rays": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int64, _vp, _vp, _vp]),
    "prr_scene_sample_light": (C.c_int, [_vp, C.c_uint64, C.c_int64, _vp, _vp, _vp, _vp]),
    "prr_env_eval": (C.c_int, [_vp, _vp, C.c_int64, _vp, _vp, _vp]),
    "prr_env_importance_sample": (C.c_int, [_vp, C.c_uint64, C.c_int64, _vp, _vp, _vp]),
    "prr_env_export": (C.c_int, [_vp, _vp, _vp, C.POINTER(C.c_float)]),
}

_lib = None


def header_symbols() -> list[str]:
    """Every function declared in include/*.h."""
    names = []
    for h in sorted(HEADER_DIR.glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        names += re.findall(r"\b(prr_\w+)\s*\(", text)
    seen = []
    for n in names:
        if n not in seen:
            seen.append(n)
    return seen


def load() -> C.CDLL:
    """Load libprr.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: run photorealisticrender4610_b200/build.py "
                          "(nvcc, sm_100a). There is no CPU fallback.")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.prr_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> int:
    if rc < 0:
        raise PrrError(rc, last_error())
    return rc
