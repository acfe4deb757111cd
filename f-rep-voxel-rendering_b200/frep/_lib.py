"""ctypes binding of the C-ABI declared in include/frep.h.

This module only loads libfrep.so and describes its structs; the user-facing
classes live in frep/__init__.py. There is no fallback: if the native library
is missing, importing fails with the build command to run.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_native" / "libfrep.so"

MAX_LEVELS = 8
MAX_LIGHTS = 8

OK, ERR_INVALID_ARG, ERR_OOM, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_UNSUPPORTED, ERR_COMPILE = range(8)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CAPACITY", 4: "TIMEOUT", 5: "CUDA",
                6: "UNSUPPORTED", 7: "COMPILE"}


class FrepError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Dag(C.Structure):
    _fields_ = [("n_nodes", C.c_uint32), ("ops", C.POINTER(C.c_uint8)), ("in0", C.POINTER(C.c_uint32)),
                ("in1", C.POINTER(C.c_uint32)), ("consts", C.POINTER(C.c_float)), ("root", C.c_uint32)]


class TapeOpts(C.Structure):
    _fields_ = [("const_reload_distance", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class TapeInfo(C.Structure):
    _fields_ = [("n_instr", C.c_uint32), ("n_slots", C.c_uint32), ("n_consts", C.c_uint32),
                ("n_minmax", C.c_uint32), ("fits_reference", C.c_uint32), ("uses_time", C.c_uint32)]


class Grid(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("dims", C.c_uint32 * MAX_LEVELS), ("low_vertex", C.c_float * 3),
                ("world_size", C.c_float)]


class BatchInfo(C.Structure):
    _fields_ = [("n_trees", C.c_uint32), ("voxelize_launches", C.c_uint32), ("upload_bytes", C.c_uint64),
                ("device_bytes", C.c_uint64), ("interval_warps_per_block", C.c_uint32),
                ("point_warps_per_block", C.c_uint32), ("root_cells_per_lane", C.c_uint32)]


class VoxelizeOpts(C.Structure):
    _fields_ = [("rounding", C.c_uint32), ("shorten", C.c_uint32), ("node_words", C.c_uint64),
                ("tape_words", C.c_uint64), ("point_cells_per_lane", C.c_uint32), ("separate_tapes", C.c_uint32)]


class TreeInfo(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("dims", C.c_uint32 * MAX_LEVELS),
                ("node_count", C.c_uint32 * MAX_LEVELS), ("node_offset", C.c_uint64 * MAX_LEVELS),
                ("node_size", C.c_uint32 * MAX_LEVELS), ("tape_size_sum", C.c_uint64 * MAX_LEVELS),
                ("tape_size_max", C.c_uint32 * MAX_LEVELS), ("node_words_used", C.c_uint64),
                ("node_words_cap", C.c_uint64), ("tape_words_used", C.c_uint64),
                ("tape_words_cap", C.c_uint64), ("overflow", C.c_uint32), ("root_tape_words", C.c_uint32)]


class CameraStruct(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3), ("up", C.c_float * 3),
                ("fov_deg", C.c_float), ("ortho_width", C.c_float), ("projection", C.c_uint32),
                ("width", C.c_uint32), ("height", C.c_uint32), ("jitter", C.c_uint32),
                ("jitter_seed", C.c_float)]


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("max_batch", C.c_uint32), ("max_inflight", C.c_uint32),
                ("interval_warps_per_block", C.c_uint32), ("point_warps_per_block", C.c_uint32)]


class RequestStruct(C.Structure):
    _fields_ = [("scene", C.c_uint64), ("camera", CameraStruct), ("tape_time", C.c_float),
                ("rgba8", C.c_void_p)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("voxelized", C.c_uint32), ("retries", C.c_uint32),
                ("latency_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "failed", "voxelized", "rerendered",
                                          "evictions", "steps", "resident_trees", "resident_bytes",
                                          "arena_bytes")] + \
               [(k, C.c_double) for k in ("p50_ms", "p99_ms", "mean_ms", "max_ms", "scenes_per_s",
                                          "max_plan_ms", "max_enqueue_ms")] + \
               [("max_step_evictions", C.c_uint64)]


class LightsStruct(C.Structure):
    _fields_ = [("count", C.c_uint32), ("direction", (C.c_float * 3) * MAX_LIGHTS),
                ("color", (C.c_float * 4) * MAX_LIGHTS), ("ambient", C.c_float * 4),
                ("background", C.c_float * 4), ("shadow_mask", C.c_uint32)]


class CompactInfo(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("dims", C.c_uint32 * MAX_LEVELS), ("mode", C.c_uint32),
                ("n_slots", C.c_uint32), ("node_count", C.c_uint32 * MAX_LEVELS),
                ("node_offset", C.c_uint64 * MAX_LEVELS), ("node_size", C.c_uint32 * MAX_LEVELS),
                ("node_words", C.c_uint64), ("tape_words", C.c_uint64), ("device_bytes", C.c_uint64)]


class AutotuneOpts(C.Structure):
    _fields_ = [("per_class", C.c_uint32), ("reps", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("margin", C.c_float), ("force", C.c_uint32), ("refine", C.c_uint32)]


class Image(C.Structure):
    _fields_ = [("rgba8", C.c_void_p), ("hits", C.c_void_p)]


HIT_DTYPE = [("t", "<f4"), ("normal", "<f4", (3,)), ("level", "<u4"), ("node", "<u4"),
             ("cell", "<u4"), ("steps", "<u4")]

_P = C.c_void_p
_SIGS = {
    "frep_last_error": (C.c_char_p, []),
    "frep_version": (C.c_char_p, []),
    "frep_tape_compile": (C.c_int, [C.POINTER(Dag), C.POINTER(_P)]),
    "frep_tape_compile_opts": (C.c_int, [C.POINTER(Dag), C.POINTER(TapeOpts), C.POINTER(_P)]),
    "frep_tape_from_reference": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, C.POINTER(_P)]),
    "frep_tape_get_info": (C.c_int, [_P, C.POINTER(TapeInfo)]),
    "frep_tape_get_instrs": (C.c_int, [_P, _P, C.c_uint32]),
    "frep_tape_get_reference": (C.c_int, [_P, _P, _P]),
    "frep_tape_eval": (C.c_int, [_P, _P, C.c_uint32, _P]),
    "frep_tape_eval_device": (C.c_int, [_P, _P, _P, C.c_uint32, _P]),
    "frep_tape_eval_intervals": (C.c_int, [_P, _P, _P, C.c_uint32, C.c_float, C.c_uint32, _P]),
    "frep_tape_destroy": (None, [_P]),
    "frep_ctx_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_P)]),
    "frep_ctx_destroy": (None, [_P]),
    "frep_ctx_memory": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "frep_tree_create": (C.c_int, [_P, C.POINTER(Grid), C.POINTER(VoxelizeOpts), C.POINTER(_P)]),
    "frep_tree_destroy": (None, [_P]),
    "frep_voxelize": (C.c_int, [_P, _P, _P, C.c_float, _P]),
    "frep_voxelize_reuse": (C.c_int, [_P, _P, _P, _P, C.c_float, _P]),
    "frep_voxelize_static_scratch": (C.c_int, [_P, _P, _P, C.c_float, _P]),
    "frep_tree_sync": (C.c_int, [_P, C.POINTER(TreeInfo)]),
    "frep_tree_work": (C.c_int, [_P, _P]),
    "frep_tree_fp32_ops": (C.c_int, [_P, _P]),
    "frep_tree_set_profiling": (C.c_int, [_P, C.c_int]),
    "frep_tree_timings": (C.c_int, [_P, _P]),
    "frep_tree_copy_nodes": (C.c_int, [_P, _P, C.c_uint64]),
    "frep_tree_copy_tapes": (C.c_int, [_P, _P, C.c_uint64]),
    "frep_lights_default": (C.c_int, [C.POINTER(LightsStruct)]),
    "frep_batch_create": (C.c_int, [_P, _P, C.c_uint32, C.POINTER(_P)]),
    "frep_batch_destroy": (None, [_P]),
    "frep_batch_voxelize": (C.c_int, [_P, _P, _P, _P]),
    "frep_batch_render": (C.c_int, [_P, _P, C.POINTER(LightsStruct), _P, _P, _P]),
    "frep_batch_run": (C.c_int, [_P, _P, _P, _P, C.POINTER(LightsStruct), _P, C.c_int, _P]),
    "frep_batch_set_profiling": (C.c_int, [_P, C.c_int]),
    "frep_batch_set_trees": (C.c_int, [_P, _P, C.c_uint32]),
    "frep_tape_from_wide": (C.c_int, [_P, C.c_uint32, C.POINTER(_P)]),
    "frep_resolve_layers": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P]),
    "frep_render_temporal": (C.c_int, [_P, _P, C.POINTER(CameraStruct), C.POINTER(LightsStruct), C.c_float,
                                       C.c_uint32, _P, _P, _P]),
    "frep_server_create": (C.c_int, [_P, C.POINTER(ServerConfig), C.POINTER(LightsStruct), C.POINTER(_P)]),
    "frep_server_destroy": (None, [_P]),
    "frep_server_add_scene": (C.c_int, [_P, _P, C.POINTER(Grid), C.POINTER(VoxelizeOpts), C.POINTER(C.c_uint64)]),
    "frep_server_submit": (C.c_int, [_P, C.POINTER(RequestStruct), C.POINTER(C.c_uint64)]),
    "frep_server_poll": (C.c_int, [_P, C.c_uint64, C.POINTER(RequestStatus)]),
    "frep_server_wait": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.POINTER(RequestStatus)]),
    "frep_server_drain": (C.c_int, [_P, C.c_uint32]),
    "frep_server_release": (C.c_int, [_P, C.c_uint64]),
    "frep_server_get_stats": (C.c_int, [_P, C.c_int, C.POINTER(ServerStats)]),
    "frep_batch_render_frames": (C.c_int, [_P, _P, C.c_uint32, _P, C.POINTER(LightsStruct), _P, _P, _P]),
    "frep_batch_set_tuning": (C.c_int, [_P, C.c_uint32, C.c_uint32]),
    "frep_batch_get_info": (C.c_int, [_P, C.POINTER(BatchInfo)]),
    "frep_batch_timings": (C.c_int, [_P, _P]),
    "frep_render": (C.c_int, [_P, _P, C.POINTER(CameraStruct), C.POINTER(LightsStruct), C.c_float,
                              C.POINTER(Image), _P]),
    "frep_tree_compact": (C.c_int, [_P, _P, C.c_uint32, _P, C.POINTER(_P)]),
    "frep_compact_get_info": (C.c_int, [_P, C.POINTER(CompactInfo)]),
    "frep_compact_destroy": (None, [_P]),
    "frep_render_compact": (C.c_int, [_P, _P, C.POINTER(CameraStruct), C.POINTER(LightsStruct), C.c_float,
                                      C.POINTER(Image), _P]),
    "frep_compact_export": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "frep_compact_check": (C.c_int, [_P, C.c_uint64]),
    "frep_compact_import": (C.c_int, [_P, _P, C.c_uint64, C.POINTER(_P)]),
    "frep_fit_pools": (C.c_int, [_P, _P, _P, _P, C.c_uint32, C.c_float, _P, _P]),
    "frep_tuning_create": (C.c_int, [C.POINTER(_P)]),
    "frep_tuning_destroy": (None, [_P]),
    "frep_tuning_load": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "frep_tuning_save": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "frep_tuning_lookup": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), _P,
                                     C.POINTER(C.c_uint32)]),
    "frep_tuning_warps": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "frep_batch_autotune": (C.c_int, [_P, _P, _P, _P, C.c_uint32, C.POINTER(LightsStruct), _P, C.c_float,
                                      C.POINTER(AutotuneOpts), _P]),
}


def load(path: Path | str = LIB_PATH) -> C.CDLL:
    path = Path(path)
    if not path.exists():
        raise ImportError(
            f"native library {path} is missing; build it with "
            f"`python f-rep-voxel-rendering_b200/frep/_build.py` (nvcc, sm_100a)")
    lib = C.CDLL(str(path))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib


def check(status: int) -> None:
    if status != OK:
        msg = lib().frep_last_error().decode(errors="replace")
        raise FrepError(status, msg)
