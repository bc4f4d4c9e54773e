"""ctypes bindings of libbt_gpu.so (include/bt_gpu.h).

The library is built in-tree by ``beamtrace2007_b200.build``; loading fails
loudly when it is missing -- there is no CPU path behind these calls.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libbt_gpu.so")

BT_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of memory", -4: "capacity exceeded",
          -5: "round limit", -6: "no CUDA device", -7: "busy", -8: "size over limit"}


class BtError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Camera(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("fwd", C.c_float * 3), ("right", C.c_float * 3), ("down", C.c_float * 3),
                ("half_w", C.c_float), ("half_h", C.c_float), ("W", C.c_int32), ("H", C.c_int32)]

    def as_array(self) -> np.ndarray:
        """eye fwd right down half_w half_h as 14 doubles (the oracle's camera form)."""
        return np.array(list(self.eye) + list(self.fwd) + list(self.right) + list(self.down) +
                        [self.half_w, self.half_h], np.float64)


class AreaLight(C.Structure):
    _fields_ = [("c", C.c_float * 3), ("U", C.c_float * 3), ("V", C.c_float * 3)]

    @staticmethod
    def from_array(a) -> "AreaLight":
        a = np.asarray(a, np.float32).ravel()
        L = AreaLight()
        for i in range(3):
            L.c[i], L.U[i], L.V[i] = a[i], a[3 + i], a[6 + i]
        return L


class SceneDesc(C.Structure):
    _fields_ = [("pos", C.c_void_p), ("num_verts", C.c_int64), ("tris", C.c_void_p), ("tri_normals", C.c_void_p),
                ("num_tris", C.c_int64), ("bounds", C.c_float * 6)]


class KdDesc(C.Structure):
    _fields_ = [("split", C.c_void_p), ("data", C.c_void_p), ("offset", C.c_void_p), ("parent", C.c_void_p),
                ("node_box", C.c_void_p), ("num_nodes", C.c_int64), ("tri_indices", C.c_void_p),
                ("num_refs", C.c_int64), ("bounds", C.c_float * 6)]


class KdParams(C.Structure):
    _fields_ = [("cost_traverse", C.c_float), ("cost_intersect", C.c_float), ("empty_bonus", C.c_float),
                ("max_depth", C.c_int32), ("bin_threshold", C.c_int32), ("bins", C.c_int32),
                ("clip_bounds", C.c_int32), ("single_leaf", C.c_int32)]


class SceneFileInfo(C.Structure):
    _fields_ = [("name", C.c_char * 128), ("num_verts", C.c_int64), ("num_tris", C.c_int64),
                ("num_materials", C.c_int64), ("num_views", C.c_int64), ("cull_backfaces", C.c_int32),
                ("has_point_light", C.c_int32), ("has_area_light", C.c_int32), ("up", C.c_float * 3),
                ("point_light", C.c_float * 3), ("light_c", C.c_float * 3), ("light_u", C.c_float * 3),
                ("light_v", C.c_float * 3), ("light_intensity", C.c_float), ("background", C.c_float * 3)]


class GpuInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("sm_count", C.c_int32), ("mem_gb", C.c_double), ("cc_major", C.c_int32),
                ("cc_minor", C.c_int32)]


class GpuConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("budget", C.c_int32), ("primary_budget", C.c_int32),
                ("capacity", C.c_int64), ("blocks_per_sm", C.c_int32), ("kernel_timing", C.c_int32),
                ("max_retries", C.c_int32), ("tail_records", C.c_int64),
                ("eps_stats", C.c_int32), ("yield_pct", C.c_int32),
                ("fuse_primary", C.c_int32), ("eps_fp64", C.c_int32),
                ("graph_rounds", C.c_int32), ("trace_ctas", C.c_int32)]


class SoftOpts(C.Structure):
    _fields_ = [("exact", C.c_int32), ("offset", C.c_float)]


class SoftJob(C.Structure):
    _fields_ = [("cam", Camera), ("light", AreaLight), ("opts", SoftOpts), ("d_tri", C.c_void_p),
                ("d_vis", C.c_void_p), ("d_E", C.c_void_p), ("d_Eu", C.c_void_p), ("scene", C.c_int32)]


class RunInfo(C.Structure):
    _fields_ = [("kd_steps", C.c_uint64), ("leaf_visits", C.c_uint64), ("tri_tests", C.c_uint64),
                ("hits", C.c_uint64), ("splits", C.c_uint64), ("beams", C.c_uint64), ("root_beams", C.c_uint64),
                ("presplit_beams", C.c_uint64), ("five_splits", C.c_uint64), ("climbs", C.c_uint64),
                ("dropped_area", C.c_double), ("eps_band_corners", C.c_uint64), ("eps_fp64_flips", C.c_uint64),
                ("ms_primary", C.c_double), ("ms_trace", C.c_double), ("ms_total", C.c_double),
                ("ms_round", C.c_double), ("launches", C.c_int32), ("round_launches", C.c_int32),
                ("passes", C.c_int32), ("retried_roots", C.c_int32), ("max_spill", C.c_int32),
                ("roots", C.c_int64), ("rounds", C.c_int32), ("tail_rounds", C.c_int32), ("ms_kernel_admit", C.c_double),
                ("ms_kernel_trace", C.c_double), ("ms_kernel_clip", C.c_double), ("yields", C.c_int64),
                ("overflow_roots", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Polys(C.Structure):
    _fields_ = [("x", C.c_void_p), ("y", C.c_void_p), ("n", C.c_void_p), ("tri", C.c_void_p), ("area", C.c_void_p),
                ("root", C.c_void_p), ("cap", C.c_int64)]


BT_REQ_SOFT, BT_REQ_PRIMARY_IDS, BT_REQ_POINT_MASK = 0, 1, 2


class Request(C.Structure):
    _fields_ = [("kind", C.c_int32), ("scene", C.c_int32), ("cam", Camera), ("light", AreaLight), ("opts", SoftOpts),
                ("point_light", C.c_float * 3), ("cull", C.c_int32), ("tile", C.c_int32), ("tri", C.c_void_p),
                ("vis", C.c_void_p), ("E", C.c_void_p), ("Eu", C.c_void_p), ("mask", C.c_void_p),
                ("user", C.c_uint64)]


class Completion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("user", C.c_uint64), ("kind", C.c_int32), ("status", C.c_int32),
                ("ms_queued", C.c_double), ("ms_total", C.c_double), ("error", C.c_char * 160)]


class ServeConfig(C.Structure):
    _fields_ = [("vis_lanes", C.c_int32), ("soft_jobs", C.c_int32), ("soft_pixels", C.c_int64),
                ("capacity", C.c_int64), ("fold_ms", C.c_double), ("memory_budget", C.c_int64),
                ("soft_blocks_per_sm", C.c_int32)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("refused", C.c_int64), ("queued", C.c_int64),
                ("running", C.c_int64), ("soft_runs", C.c_int64), ("soft_folded", C.c_int64),
                ("scene_bytes", C.c_int64), ("lane_bytes", C.c_int64), ("queue_high_water", C.c_int64),
                ("admitted_bytes", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = C.c_void_p
_I = C.c_int
_I64 = C.c_int64

# name -> (restype, argtypes)
SIGNATURES = {
    "bt_gpu_last_error": (C.c_char_p, []),
    "bt_gpu_config_default": (None, [C.POINTER(GpuConfig)]),
    "bt_scene_finalize": (_I64, [_P, _I64, _P, _I64, _P, _P, _P, _P]),
    "bt_kd_params_default": (None, [C.POINTER(KdParams)]),
    "bt_kd_build": (_I, [_P, _P, _P, _I64, _P, C.POINTER(KdParams), C.POINTER(_P)]),
    "bt_kd_sizes": (None, [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "bt_kd_view": (None, [_P, C.POINTER(KdDesc)]),
    "bt_kd_free": (None, [_P]),
    "bt_kd_build_gpu": (_I, [_P, _I64, _P, _P, _I64, _P, C.POINTER(KdParams), C.c_int32, C.POINTER(_P),
                             C.POINTER(C.c_double)]),
    "bt_scene_load_config": (_I, [C.c_char_p, C.POINTER(_P)]),
    "bt_scene_parse_config": (_I, [C.c_char_p, C.POINTER(_P)]),
    "bt_scene_file_info_get": (None, [_P, C.POINTER(SceneFileInfo)]),
    "bt_scene_file_arrays": (None, [_P, _P, _P, _P, _P, _P]),
    "bt_scene_file_free": (None, [_P]),
    "bt_camera_make": (None, [_P, _P, C.c_float, _P, C.c_int32, C.c_int32, C.POINTER(Camera)]),
    "bt_gpu_available": (_I, [C.POINTER(GpuInfo)]),
    "bt_gpu_create": (_I, [C.POINTER(SceneDesc), C.POINTER(KdDesc), C.POINTER(GpuConfig), C.POINTER(_P)]),
    "bt_gpu_destroy": (_I, [_P]),
    "bt_gpu_add_scene": (_I, [_P, C.POINTER(SceneDesc), C.POINTER(KdDesc), C.POINTER(C.c_int32)]),
    "bt_gpu_soft": (_I, [_P, C.POINTER(Camera), C.POINTER(AreaLight), C.POINTER(SoftOpts), _P, _P, _P, _P,
                         C.POINTER(RunInfo)]),
    "bt_gpu_soft_points": (_I, [_P, C.POINTER(AreaLight), C.POINTER(SoftOpts), _I64, _P, _P, _P, _P, _P, _P,
                                C.POINTER(RunInfo)]),
    "bt_gpu_soft_points_device": (_I, [_P, C.POINTER(AreaLight), C.POINTER(SoftOpts), _I64, _P, _P, _P, _P, _P,
                                       _P, C.POINTER(RunInfo)]),
    "bt_gpu_soft_points_noalloc": (_I, [C.POINTER(SceneDesc), C.POINTER(KdDesc), C.POINTER(AreaLight),
                                        C.POINTER(SoftOpts), _I64, _P, _P, _P, _P, _P, _P, C.POINTER(RunInfo)]),
    "bt_gpu_soft_device": (_I, [_P, C.POINTER(Camera), C.POINTER(AreaLight), C.POINTER(SoftOpts), _P, _P, _P, _P,
                                C.POINTER(RunInfo)]),
    "bt_gpu_batch_soft": (_I, [_P, C.c_int32, C.POINTER(SoftJob), C.POINTER(RunInfo)]),
    "bt_gpu_primary_rays": (_I, [_P, C.POINTER(Camera), _P, _P, _P]),
    "bt_gpu_primary_rays_device": (_I, [_P, C.POINTER(Camera), _P, _P, _P]),
    "bt_gpu_primary": (_I, [_P, C.POINTER(Camera), C.c_int32, C.c_int32, C.POINTER(Polys), C.POINTER(_I64),
                            C.POINTER(RunInfo)]),
    "bt_gpu_point": (_I, [_P, C.POINTER(Camera), C.POINTER(Polys), _I64, _P, C.POINTER(Polys), C.POINTER(_I64),
                          C.POINTER(RunInfo)]),
    "bt_gpu_primary_ids": (_I, [_P, C.POINTER(Camera), C.c_int32, C.c_int32, _P, C.POINTER(RunInfo)]),
    "bt_gpu_primary_ids_device": (_I, [_P, C.POINTER(Camera), C.c_int32, C.c_int32, _P, C.POINTER(RunInfo)]),
    "bt_gpu_point_mask": (_I, [_P, C.POINTER(Camera), C.c_int32, C.c_int32, _P, _P, _P, C.POINTER(RunInfo)]),
    "bt_gpu_point_mask_device": (_I, [_P, C.POINTER(Camera), C.c_int32, C.c_int32, _P, _P, _P,
                                      C.POINTER(RunInfo)]),
    "bt_gpu_raster": (_I, [_P, C.POINTER(Camera), C.POINTER(Polys), _I64, C.POINTER(Polys), _I64, _P, _P]),
    "bt_gpu_last_polys": (_I, [_P, C.POINTER(Polys), C.POINTER(_I64)]),
    "bt_gpu_serve_start": (_I, [_P, C.POINTER(ServeConfig)]),
    "bt_gpu_submit": (_I, [_P, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "bt_gpu_poll": (_I, [_P, C.POINTER(Completion), C.c_int32, C.POINTER(C.c_int32), C.c_int32]),
    "bt_gpu_serve_stats": (_I, [_P, C.POINTER(ServeStats)]),
}

_lib = None


def lib():
    """Loads libbt_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m beamtrace2007_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(code: int):
    if code != BT_OK:
        raise BtError(code, lib().bt_gpu_last_error().decode(errors="replace"))
    return code


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
