"""ctypes binding of libvkpt_cuda (include/vkptc.h).

The library is built in-tree (vkpathtracer_b200/_lib/libvkpt_cuda.so).  There
is no fallback: if the library is missing or has no CUDA device, loading or
creating a context raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libvkpt_cuda.so")

STATUS_NAMES = ["Ok", "Unsupported", "InvalidArgument", "NotReady", "Busy", "AllocFailed", "Timeout",
                "Cancelled", "InternalError"]
OK, UNSUPPORTED, INVALID_ARGUMENT, NOT_READY, BUSY, ALLOC_FAILED, TIMEOUT, CANCELLED, INTERNAL_ERROR = range(9)
LIFECYCLE_NAMES = ["uninitialized", "configured", "scene_loaded", "ready", "failed"]
QUERY_CLOSEST, QUERY_ANY = 0, 1


class Config(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("block_size", ctypes.c_uint32), ("stack_depth", ctypes.c_uint32),
                ("math_mode", ctypes.c_uint32), ("collect_stats", ctypes.c_uint32), ("wave_paths", ctypes.c_uint32),
                ("stage_timing", ctypes.c_uint32), ("steps", ctypes.c_uint32), ("bvh_mode", ctypes.c_uint32),
                ("build_mode", ctypes.c_uint32), ("triangle_test", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 2)]


BVH_REFERENCE, BVH_SAH = 0, 1
BUILD_DEVICE, BUILD_HOST = 0, 1
TRIANGLE_MT, TRIANGLE_WATERTIGHT = 0, 1
ACCEL_WIDE_NODES, ACCEL_TRIANGLES, ACCEL_TIE_NODES, ACCEL_SHADING = range(4)


class RenderSettingsC(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("spp", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("seed", ctypes.c_uint64), ("enable_nee", ctypes.c_uint32),
                ("enable_mis", ctypes.c_uint32), ("deterministic", ctypes.c_uint32),
                ("rr_start_depth", ctypes.c_uint32), ("rr_min_survival", ctypes.c_float),
                ("rr_max_survival", ctypes.c_float), ("camera_aperture_radius", ctypes.c_float),
                ("camera_focus_distance", ctypes.c_float), ("firefly_clamp", ctypes.c_float),
                ("reserved", ctypes.c_uint32)]


class SceneView(ctypes.Structure):
    _fields_ = [("vertices", ctypes.c_void_p), ("vertex_count", ctypes.c_uint32),
                ("indices", ctypes.c_void_p), ("index_count", ctypes.c_uint32),
                ("instances", ctypes.c_void_p), ("instance_count", ctypes.c_uint32),
                ("materials", ctypes.c_void_p), ("material_count", ctypes.c_uint32),
                ("lights", ctypes.c_void_p), ("light_count", ctypes.c_uint32),
                ("environment", ctypes.c_float * 3), ("camera_position", ctypes.c_float * 3),
                ("camera_target", ctypes.c_float * 3), ("camera_up", ctypes.c_float * 3),
                ("camera_fov_deg", ctypes.c_float), ("camera_aperture_radius", ctypes.c_float),
                ("camera_focus_distance", ctypes.c_float), ("environment_map", ctypes.c_void_p),
                ("environment_map_width", ctypes.c_uint32), ("environment_map_height", ctypes.c_uint32),
                ("environment_map_scale", ctypes.c_float * 3),
                ("sdf_primitives", ctypes.c_void_p), ("sdf_count", ctypes.c_uint32),
                ("instance_local", ctypes.c_void_p), ("instance_transforms", ctypes.c_void_p),
                ("local_vertices", ctypes.c_void_p), ("local_vertex_count", ctypes.c_uint32),
                ("local_indices", ctypes.c_void_p), ("local_index_count", ctypes.c_uint32),
                ("camera_lens_set", ctypes.c_uint32), ("camera_iris_blade_count", ctypes.c_uint32),
                ("camera_iris_rotation_degrees", ctypes.c_float), ("camera_iris_roundness", ctypes.c_float),
                ("camera_anamorphic_squeeze", ctypes.c_float)]

# vkptc_sdf_shape
SDF_SPHERE, SDF_BOX, SDF_ROUNDED_BOX, SDF_PLANE, SDF_TORUS, SDF_CAPSULE = range(6)


class InstanceUpdate(ctypes.Structure):
    _fields_ = [("instance_index", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("translation", ctypes.c_float * 3),
                ("rotation", ctypes.c_float * 4), ("scale", ctypes.c_float * 3)]


class CameraC(ctypes.Structure):
    """vkptc_camera: the RTCameraState fields the render reads."""
    _fields_ = [("position", ctypes.c_float * 3), ("target", ctypes.c_float * 3), ("up", ctypes.c_float * 3),
                ("fov_deg", ctypes.c_float), ("aperture_radius", ctypes.c_float), ("focus_distance", ctypes.c_float),
                ("iris_blade_count", ctypes.c_uint32), ("iris_rotation_degrees", ctypes.c_float),
                ("iris_roundness", ctypes.c_float), ("anamorphic_squeeze", ctypes.c_float)]


class SceneDelta(ctypes.Structure):
    """vkptc_scene_delta: RTSceneDeltaUpdate with instances resolved to indices."""
    _fields_ = [("material_indices", ctypes.c_void_p), ("materials", ctypes.c_void_p),
                ("material_count", ctypes.c_uint32),
                ("light_indices", ctypes.c_void_p), ("lights", ctypes.c_void_p), ("light_count", ctypes.c_uint32),
                ("instance_indices", ctypes.c_void_p), ("instance_material_indices", ctypes.c_void_p),
                ("instance_material_count", ctypes.c_uint32),
                ("environment_changed", ctypes.c_uint32), ("environment", ctypes.c_float * 3)]


class FilmResolve(ctypes.Structure):
    _fields_ = [("exposure", ctypes.c_float), ("white_balance_kelvin", ctypes.c_float), ("tone_map", ctypes.c_uint32),
                ("output_transform", ctypes.c_uint32), ("gamma", ctypes.c_float), ("clamp_output", ctypes.c_uint32)]


TONE_MAPS = {"linear": 0, "reinhard": 1, "filmic": 2, "aces": 3}
OUTPUT_TRANSFORMS = {"gamma": 0, "linear": 1}
READBACK_INVALID, READBACK_PENDING, READBACK_READY, READBACK_FAILED = range(4)


class BvhView(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_void_p), ("node_count", ctypes.c_uint32),
                ("prim_indices", ctypes.c_void_p), ("prim_count", ctypes.c_uint32)]


class Tile(ctypes.Structure):
    _fields_ = [("x", ctypes.c_uint32), ("y", ctypes.c_uint32), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("sample_index", ctypes.c_uint32), ("tile_id", ctypes.c_uint32),
                ("gpu_id", ctypes.c_uint32)]


class Counters(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("samples", "rays", "triangle_tests", "sdf_tests", "sdf_steps",
                                                "triangle_hits", "sdf_hits", "sdf_misses", "bvh_node_visits",
                                                "bvh_leaf_visits", "shadow_tests")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class TracerStatusC(ctypes.Structure):
    _fields_ = [("lifecycle", ctypes.c_uint32), ("scene_loaded", ctypes.c_uint32), ("accel_valid", ctypes.c_uint32),
                ("ready_to_render", ctypes.c_uint32), ("current_sample", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("last_sample_us", ctypes.c_uint64),
                ("total_samples", ctypes.c_uint64), ("accumulation_gen", ctypes.c_uint64)]


class AccelInfo(ctypes.Structure):
    _fields_ = [("primitive_count", ctypes.c_uint32), ("binary_node_count", ctypes.c_uint32),
                ("binary_leaf_count", ctypes.c_uint32), ("wide_node_count", ctypes.c_uint32),
                ("wide_depth", ctypes.c_uint32), ("stack_required", ctypes.c_uint32),
                ("build_ms", ctypes.c_double), ("device_bytes", ctypes.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchTuning(ctypes.Structure):
    _fields_ = [("pool_paths", ctypes.c_uint32), ("block_size", ctypes.c_uint32), ("stack_depth", ctypes.c_uint32),
                ("steps", ctypes.c_uint32), ("sample_limit", ctypes.c_uint32), ("use_graph", ctypes.c_uint32),
                ("occupancy", ctypes.c_uint32), ("barrier_spins", ctypes.c_uint32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("jobs", ctypes.c_uint32), ("graph_used", ctypes.c_uint32), ("paths", ctypes.c_uint64),
                ("segments", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("device_ms", ctypes.c_double), ("grid", ctypes.c_uint32),
                ("block", ctypes.c_uint32), ("pool_paths", ctypes.c_uint32), ("stack_depth", ctypes.c_uint32),
                ("steps", ctypes.c_uint32), ("iterations", ctypes.c_uint32),
                ("ext_rays", ctypes.c_uint64), ("ext_nodes", ctypes.c_uint64), ("ext_tris", ctypes.c_uint64),
                ("shadow_queries", ctypes.c_uint64), ("shadow_nodes", ctypes.c_uint64),
                ("shadow_tris", ctypes.c_uint64), ("stage_ms", ctypes.c_double * 5)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_ if n not in ("reserved", "stage_ms")}
        d["stage_ms"] = dict(zip(("regen", "extend", "shade", "shadow", "finish"), list(self.stage_ms)))
        return d


class AdjointDesc(ctypes.Structure):
    _fields_ = [("spp", ctypes.c_uint32), ("first_sample", ctypes.c_uint32), ("frame", ctypes.c_uint32),
                ("backward_frame", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


ADJ_DECORRELATED = 1


class AdjointStats(ctypes.Structure):
    _fields_ = [("paths", ctypes.c_uint64), ("forwards", ctypes.c_uint64), ("backwards", ctypes.c_uint64),
                ("forward_ms", ctypes.c_double), ("backward_ms", ctypes.c_double),
                ("forward_grid", ctypes.c_uint32), ("backward_grid", ctypes.c_uint32), ("block", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


ADJ_PARAMS_PER_MATERIAL = 7
ADJ_MAX_MATERIALS = 64
ADJ_MAX_DEPTH = 8

P = ctypes.c_void_p
U32, U64, I32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32
ABI_VERSION = 2   # VKPTC_ABI_VERSION of the struct layouts above

# name -> (restype, argtypes); every symbol include/vkptc.h declares.
SIGNATURES = {
    "vkptc_abi_version": (U32, []),
    "vkptc_create": (I32, [ctypes.POINTER(Config), ctypes.POINTER(P)]),
    "vkptc_destroy": (I32, [P]),
    "vkptc_configure": (I32, [P, ctypes.POINTER(RenderSettingsC)]),
    "vkptc_load_scene": (I32, [P, ctypes.POINTER(SceneView)]),
    "vkptc_build_acceleration": (I32, [P]),
    "vkptc_load_bvh": (I32, [P, ctypes.POINTER(BvhView)]),
    "vkptc_get_accel_info": (I32, [P, ctypes.POINTER(AccelInfo)]),
    "vkptc_read_accel": (I32, [P, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "vkptc_resolve_ldr": (I32, [P, ctypes.POINTER(FilmResolve), ctypes.c_void_p]),
    "vkptc_update_instance_transforms": (I32, [P, ctypes.c_void_p, ctypes.c_uint32]),
    "vkptc_batch_read_films": (I32, [P, ctypes.c_void_p, ctypes.c_void_p]),
    "vkptc_check_instance_transforms": (I32, [P, ctypes.c_void_p, ctypes.c_uint32]),
    "vkptc_update_camera": (I32, [P, ctypes.POINTER(CameraC)]),
    "vkptc_get_camera": (I32, [P, ctypes.POINTER(CameraC)]),
    "vkptc_update_scene_delta": (I32, [P, ctypes.POINTER(SceneDelta)]),
    "vkptc_request_ldr_readback": (I32, [P, ctypes.POINTER(FilmResolve), ctypes.POINTER(ctypes.c_uint64)]),
    "vkptc_poll_ldr_readback": (I32, [P, ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32)]),
    "vkptc_measure_read_bandwidth": (I32, [P, ctypes.c_uint64, U32, ctypes.POINTER(ctypes.c_double)]),
    "vkptc_device_name": (I32, [P, ctypes.c_char_p, U32, ctypes.POINTER(U32)]),
    "vkptc_build_binary_bvh": (I32, [ctypes.POINTER(SceneView), P, ctypes.POINTER(U32), P, ctypes.POINTER(U32)]),
    "vkptc_reset": (I32, [P]),
    "vkptc_shutdown": (I32, [P]),
    "vkptc_render": (I32, [P, ctypes.POINTER(Tile), U32, U32, P]),
    "vkptc_render_frame": (I32, [P, U32, U32, U32]),
    "vkptc_synchronize": (I32, [P]),
    "vkptc_set_stream": (I32, [P, P]),
    "vkptc_read_stage_times": (I32, [P, P, P]),
    "vkptc_read_film": (I32, [P, P, P, P]),
    "vkptc_resolve_hdr": (I32, [P, P]),
    "vkptc_write_film": (I32, [P, P, P, P]),
    "vkptc_read_counters": (I32, [P, ctypes.POINTER(Counters)]),
    "vkptc_get_status": (I32, [P, ctypes.POINTER(TracerStatusC)]),
    "vkptc_read_traversal_stats": (I32, [P, P]),
    "vkptc_last_error": (ctypes.c_char_p, [P]),
    "vkptc_trace_rays": (I32, [P, P, P, U64, U32, P, P]),
    "vkptc_trace_rays_device": (I32, [P, P, P, U64, U32, P, P, P]),
    "vkptc_render_tile_noalloc": (I32, [P, ctypes.POINTER(Tile), U32, P, P, P]),
    "vkptc_batch_create": (I32, [ctypes.POINTER(Config), ctypes.POINTER(P)]),
    "vkptc_batch_destroy": (I32, [P]),
    "vkptc_batch_add_job": (I32, [P, ctypes.POINTER(SceneView), ctypes.POINTER(RenderSettingsC),
                                  ctypes.POINTER(U32)]),
    "vkptc_batch_run": (I32, [P, U32, ctypes.POINTER(BatchTuning)]),
    "vkptc_batch_read_film": (I32, [P, U32, P, P]),
    "vkptc_batch_get_stats": (I32, [P, ctypes.POINTER(BatchStats)]),
    "vkptc_batch_last_error": (ctypes.c_char_p, [P]),
    "vkptc_adjoint_setup": (I32, [P, ctypes.POINTER(AdjointDesc), P, U64]),
    "vkptc_forward": (I32, [P, P, U32, P, ctypes.POINTER(ctypes.c_double), P]),
    "vkptc_backward": (I32, [P, P, U32]),
    "vkptc_backward_weighted": (I32, [P, P, P, U32]),
    "vkptc_adjoint_set_frames": (I32, [P, U32, U32]),
    "vkptc_adjoint_read_samples": (I32, [P, P, P]),
    "vkptc_adjoint_get_stats": (I32, [P, ctypes.POINTER(AdjointStats)]),
}
BATCH_PLAIN, BATCH_PERSISTENT, BATCH_LOOP = 0, 1, 2
NOALLOC_MAX_PATHS = 65536

_LIB = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libvkpt_cuda.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"libvkpt_cuda.so is not built ({path}); run `python -m vkpathtracer_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.vkptc_abi_version() != ABI_VERSION:
        raise RuntimeError(f"libvkpt_cuda.so has ABI version {lib.vkptc_abi_version()}, these bindings {ABI_VERSION}; "
                           "rebuild it")
    _LIB = lib
    return lib


class VkptcError(RuntimeError):
    def __init__(self, code: int, message: str):
        self.code = code
        name = STATUS_NAMES[code] if 0 <= code < len(STATUS_NAMES) else str(code)
        super().__init__(f"{name}: {message}")
