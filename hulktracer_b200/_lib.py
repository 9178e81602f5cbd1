"""ctypes binding of ``libhulkcuda.so`` (the C ABI in include/hulkcuda.h).

There is no fallback: if the library is missing or a call fails, an exception
is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libhulkcuda.so")

HK_OK = 0
STATUS_NAMES = {0: "HK_OK", 1: "HK_E_ALLOC", 2: "HK_E_FILE_OPEN", 3: "HK_E_FILE_CLOSE",
                4: "HK_E_ILLEGAL_INPUT", 5: "HK_E_NODE_NOT_FOUND", 16: "HK_E_CUDA",
                17: "HK_E_DEVICE_TIMEOUT", 18: "HK_E_CAPACITY", 19: "HK_E_BOUNDS", 20: "HK_E_STATE"}

FULLSTACK, SHORTSTACK, SMEMSTACK, RESTART, RESTART_EARLY, ROPES, BRUTE = range(7)
VARIANTS = {"fullstack": FULLSTACK, "shortstack": SHORTSTACK, "smemstack": SMEMSTACK,
            "restart": RESTART, "restart_early": RESTART_EARLY, "ropes": ROPES, "brute": BRUTE}
BUILD_BINNED, BUILD_LEARNED, BUILD_SAH_RESORT = 0, 1, 2
SHADE_CPU, SHADE_PICTURE, SHADE_MIRROR = 0, 1, 2


class HkError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, str(status)), msg))
        self.status = status


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("traverse_cost", C.c_float), ("intersect_cost", C.c_float),
                ("max_depth", C.c_uint32), ("leaf_size", C.c_uint32), ("bins", C.c_uint32),
                ("short_stack", C.c_uint32), ("block_size", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("max_refs", C.c_uint32), ("topk", C.c_uint32), ("fallback_ratio", C.c_float),
                ("exact_max", C.c_uint32), ("spin_limit", C.c_uint32), ("max_steps", C.c_uint32),
                ("sah_sample", C.c_uint32), ("subtree_max", C.c_uint32),
                ("subtree_depth", C.c_uint32), ("level_streams", C.c_uint32)]


class TuneResult(C.Structure):
    _fields_ = [("variant", C.c_int), ("block_size", C.c_uint32), ("short_stack", C.c_uint32),
                ("best_ms", C.c_float), ("default_ms", C.c_float), ("tried", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BuildTuneResult(C.Structure):
    _fields_ = [("subtree_max", C.c_uint32), ("subtree_depth", C.c_uint32), ("level_streams", C.c_uint32),
                ("best_ms", C.c_float),
                ("default_ms", C.c_float), ("tried", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TreeStats(C.Structure):
    _fields_ = [("nodes", C.c_uint32), ("leaves", C.c_uint32), ("refs", C.c_uint32), ("depth", C.c_uint32),
                ("build_ms", C.c_float), ("capacity_hit", C.c_uint32), ("learned_nodes", C.c_uint32),
                ("fallback_nodes", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class StreamStats(C.Structure):
    _fields_ = [("launches", C.c_uint32), ("leaves_loaded", C.c_uint32), ("leaves_evicted", C.c_uint32),
                ("resident", C.c_uint32), ("bytes_paged", C.c_uint64), ("ms", C.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AffInfo(C.Structure):
    _fields_ = [("nv", C.c_uint32), ("nt", C.c_uint32), ("nmeshes", C.c_uint32), ("ndynamic", C.c_uint32),
                ("ntransforms", C.c_uint32), ("nanimations", C.c_uint32), ("nlights", C.c_uint32),
                ("has_view", C.c_int32), ("from_", C.c_float * 3), ("at", C.c_float * 3), ("up", C.c_float * 3),
                ("fov_deg", C.c_float), ("hither", C.c_float), ("resx", C.c_int32), ("resy", C.c_int32),
                ("has_anim_params", C.c_int32), ("anim_start", C.c_float), ("anim_end", C.c_float),
                ("anim_frames", C.c_int32), ("has_camera_anim", C.c_int32)]

    def as_dict(self):
        out = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            out[k.rstrip("_")] = list(v) if hasattr(v, "__len__") else v
        return out


NOALLOC_SCRATCH_BYTES = 24 << 20
MLP_IN, MLP_HID, MLP_OUT = 200, 256, 96
MLP_PARAMS = 200 * 256 + 256 + 2 * (256 * 256 + 256) + 256 * 96 + 96

HIT_DTYPE = np.dtype([("t", np.float32), ("tri", np.int32)])

_lib = None


def load(path: str = LIB_PATH):
    """Load the CUDA library (raises if it is absent: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError("libhulkcuda.so not built (%s); run python -m hulktracer_b200.build" % path)
    L = C.CDLL(path)
    vp, u32, f32p, u32p = C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p
    sig = {
        "hk_config_default": [C.POINTER(Config)],
        "hk_create": [C.POINTER(C.c_void_p), C.POINTER(Config)],
        "hk_destroy": [vp],
        "hk_set_stream": [vp, vp],
        "hk_synchronize": [vp],
        "hk_scene_upload": [vp, f32p, u32, u32p, u32],
        "hk_scene_set_box": [vp, f32p],
        "hk_scene_get_box": [vp, f32p],
        "hk_scene_set_parts": [vp, u32p, u32],
        "hk_scene_transform": [vp, f32p],
        "hk_scene_get_vertices": [vp, f32p],
        "hk_scene_get_counts": [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "hk_tree_save_file": [vp, C.c_char_p],
        "hk_obj_parse": [C.c_char_p, f32p, u32, vp, u32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "hk_scene_load_obj": [vp, C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "hk_set_frame_shading": [vp, C.c_int],
        "hk_tree_load_file": [vp, C.c_char_p, C.c_int],
        "hk_scene_set_mirrors": [vp, vp, u32],
        "hk_precompute": [vp],
        "hk_cache_import": [vp, f32p, u32],
        "hk_cache_export": [vp, f32p],
        "hk_build": [vp, C.c_int, C.POINTER(TreeStats)],
        "hk_tree_import": [vp, u32p, u32, u32p, u32],
        "hk_tree_export": [vp, u32p, u32, u32p, u32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "hk_tree_export_compact": [vp, u32p, u32, u32p, u32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "hk_tree_stats_get": [vp, C.POINTER(TreeStats)],
        "hk_tree_cost": [vp, C.c_double, C.c_double, C.POINTER(C.c_double)],
        "hk_build_level_counts": [vp, u32p, u32p, u32, C.POINTER(C.c_uint32)],
        "hk_build_subtree_counts": [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)],
        "hk_trace": [vp, f32p, u32, C.c_int, vp],
        "hk_trace_device": [vp, vp, u32, C.c_int, vp],
        "hk_set_counting": [vp, C.c_int],
        "hk_get_counters": [vp, vp],
        "hk_camera_rays": [vp, f32p, u32, u32, f32p],
        "hk_render": [vp, f32p, f32p, u32, u32, u32, C.c_int, C.c_int, u32p],
        "hk_render_device": [vp, f32p, f32p, u32, u32, u32, C.c_int, C.c_int, vp],
        "hk_render_rows_device": [vp, f32p, f32p, u32, u32, u32, u32, u32, C.c_int, C.c_int, vp],
        "hk_shade_picture": [vp, f32p, f32p, u32, f32p, u32, u32p],
        "hk_frame": [vp, f32p, f32p, f32p, u32, u32, u32, C.c_int, C.c_int, C.c_int, vp, C.POINTER(TreeStats)],
        "hk_get_ray_counts": [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
        "hk_frame_graph_info": [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
        "hk_render_noalloc": [vp, vp, vp, u32, f32p, f32p, f32p, u32, u32, u32, C.c_int, vp, vp],
        "hk_autotune": [vp, vp, u32, C.c_char_p, C.POINTER(TuneResult)],
        "hk_autotune_build": [vp, C.c_int, u32, C.POINTER(BuildTuneResult)],
        "hk_set_build_layout": [vp, u32, u32, u32],
        "hk_set_trace_config": [vp, u32, u32],
        "hk_mlp_init": [vp, C.c_uint64],
        "hk_mlp_save": [vp, C.c_char_p],
        "hk_mlp_load": [vp, C.c_char_p],
        "hk_mlp_get_params": [vp, f32p, u32],
        "hk_mlp_set_params": [vp, f32p, u32],
        "hk_mlp_forward": [vp, f32p, u32, f32p],
        "hk_mlp_grad": [vp, f32p, vp, u32, f32p, vp],
        "hk_mlp_record": [vp, u32],
        "hk_mlp_dataset": [vp, f32p, vp, u32, C.POINTER(C.c_uint32)],
        "hk_mlp_train": [vp, u32, u32, C.c_float, C.c_uint64, f32p],
        "hk_set_proposal_log": [vp, C.c_int],
        "hk_set_debug_flags": [vp, u32],
        "hk_get_proposal_log": [vp, vp, u32, C.POINTER(C.c_uint32)],
        "hk_batch_create": [vp, C.POINTER(C.c_void_p)],
        "hk_batch_destroy": [vp],
        "hk_batch_add_scene": [vp, f32p, u32, u32p, u32, C.POINTER(C.c_uint32)],
        "hk_batch_trace_device": [vp, vp, u32p, u32, C.c_int, vp, f32p],
        "hk_stream_setup": [vp, u32],
        "hk_trace_streamed": [vp, f32p, u32, vp, C.POINTER(StreamStats)],
        "hk_aff_open": [C.c_char_p, C.POINTER(C.c_void_p)],
        "hk_aff_close": [vp],
        "hk_aff_get_info": [vp, C.POINTER(AffInfo)],
        "hk_aff_geometry": [vp, f32p, u32p, u32p],
        "hk_aff_part_matrices": [vp, C.c_float, f32p],
        "hk_aff_lights": [vp, f32p],
        "hk_aff_camera": [vp, C.c_float, f32p],
        "hk_scene_load_aff": [vp, vp, C.c_float],
        "hk_scene_animate_aff": [vp, vp, C.c_float],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.hk_last_error.argtypes = [vp]
    L.hk_last_error.restype = C.c_char_p
    L.hk_aff_last_error.argtypes = []
    L.hk_aff_last_error.restype = C.c_char_p
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names the header declares (used by the load test)."""
    import re
    hdr = os.path.join(os.path.dirname(PKG), "include", "hulkcuda.h")
    txt = open(hdr).read()
    return sorted(set(re.findall(r"^(?:hk_status|const char \*)\s*(hk_\w+)\s*\(", txt, re.M)))


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
