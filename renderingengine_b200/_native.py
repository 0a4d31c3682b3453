"""ctypes binding of the C ABI declared in include/re_b200.h.

Loading fails loudly when the sm_100a library has not been built: there is no
CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "_lib" / "libre_b200.so"

# ---------------------------------------------------------------------------
# Record dtypes, byte-compatible with the reference contracts (see re_b200.h).
# ---------------------------------------------------------------------------
TRIANGLE_DTYPE = np.dtype([
    ("positions", "<f4", (3, 4)), ("normals", "<f4", (3, 4)), ("texcoords", "<f4", (3, 4)),
    ("identity", "<u4", 4), ("metadata", "<u4", 4)])
NODE_DTYPE = np.dtype([("bounds_min", "<f4", 4), ("bounds_max", "<f4", 4), ("links", "<u4", 4)])
# SceneAbiV0 object-space records (contracts/SceneAbiV0.hpp:77-112).
VERTEX_V0_DTYPE = np.dtype([("position", "<f4", 4), ("normal", "<f4", 4), ("tangent", "<f4", 4),
                            ("texcoord0", "<f4", 4)])
GEOMETRY_V0_DTYPE = np.dtype([("index_range", "<u4", 4), ("identity", "<u4", 4), ("local_bounds_min", "<f4", 4),
                              ("local_bounds_max", "<f4", 4)])
INSTANCE_V0_DTYPE = np.dtype([("object_to_world", "<f4", (4, 4)), ("world_to_object", "<f4", (4, 4)),
                              ("previous_object_to_world", "<f4", (4, 4)), ("metadata", "<u4", 4),
                              ("reserved0", "<u4", 4)])
MATERIAL_V0_DTYPE = np.dtype([("base_color_factor", "<f4", 4), ("emissive_factor_strength", "<f4", 4),
                              ("surface_params", "<f4", 4), ("transmission_params", "<f4", 4),
                              ("attenuation_color_distance", "<f4", 4), ("texture_image_indices", "<u4", 4),
                              ("texture_sampler_indices", "<u4", 4), ("metadata", "<u4", 4)])
INSTANCE_FLAG_VISIBLE = 1
RAY_DTYPE = np.dtype([("origin_tmin", "<f4", 4), ("direction_tmax", "<f4", 4),
                      ("identity", "<u4", 4), ("rng", "<u4", 4)])
HIT_DTYPE = np.dtype([("position_t", "<f4", 4), ("geometric_normal_bary_u", "<f4", 4),
                      ("shading_normal_bary_v", "<f4", 4), ("ids", "<u4", 4),
                      ("metadata", "<u4", 4), ("reserved0", "<u4", 4)])
MATERIAL_DTYPE = np.dtype([
    ("base_color_metallic", "<f4", 4), ("emissive_roughness", "<f4", 4),
    ("transmission_ior", "<f4", 4), ("attenuation_color_distance", "<f4", 4),
    ("f0", "<f4", 4), ("conductor_eta", "<f4", 4), ("conductor_k", "<f4", 4),
    ("metadata", "<u4", 4)])
LIGHT_DTYPE = np.dtype([
    ("position_range", "<f4", 4), ("direction_cos_outer", "<f4", 4), ("radiance_scale", "<f4", 4),
    ("shape_params", "<f4", 4), ("identity", "<u4", 4), ("payload", "<u4", 4)])
assert TRIANGLE_DTYPE.itemsize == 176 and NODE_DTYPE.itemsize == 48
assert RAY_DTYPE.itemsize == 64 and HIT_DTYPE.itemsize == 96
assert MATERIAL_DTYPE.itemsize == 128 and LIGHT_DTYPE.itemsize == 96
# SVGF records: GBufferPixel (bools folded into flags) and SignalPixel.
GBUFFER_DTYPE = np.dtype([
    ("linear_depth", "<f4"), ("world_normal", "<f4", 3), ("diffuse_albedo", "<f4", 3),
    ("specular_albedo", "<f4", 3), ("expected_previous_linear_depth", "<f4"), ("motion", "<f4", 2),
    ("material_id", "<u4"), ("object_id", "<u4"), ("flags", "<u4")])
SIGNAL_DTYPE = np.dtype([("diffuse", "<f4", 3), ("specular", "<f4", 3)])
assert GBUFFER_DTYPE.itemsize == 64 and SIGNAL_DTYPE.itemsize == 24
GBUFFER_VALID, GBUFFER_MOTION_VALID = 1, 2
# re_lbvh_node (allocation-free LBVH build).
LBVH_NODE_DTYPE = np.dtype([("bounds_min", "<f4", 3), ("left", "<u4"), ("bounds_max", "<f4", 3), ("right", "<u4")])
LBVH_STATIC_MAX_TRIANGLES = 65536
LBVH_CHILD_LEAF = 1 << 31

# Status codes (re_status).
SUCCESS, INVALID_ARGUMENT, UNSUPPORTED, MISSING_SCENE, RECORDING_FAILED = 0, 1, 2, 3, 4
CUDA_ERROR, OUT_OF_MEMORY, FATAL_QUEUE, BUDGET_EXCEEDED, NOT_READY, TIMEOUT = 5, 6, 7, 8, 9, 10
STATUS_NAMES = {0: "Success", 1: "InvalidArgument", 2: "Unsupported", 3: "MissingScene",
                4: "RecordingFailed", 5: "CudaError", 6: "OutOfMemory", 7: "FatalQueue",
                8: "BudgetExceeded", 9: "NotReady", 10: "Timeout"}

MEMORY_HOST, MEMORY_DEVICE = 0, 1
BUILD_FLATTENED_SAH, BUILD_LBVH = 0, 1
HIT_KIND_MISS, HIT_KIND_TRIANGLE, HIT_KIND_INVALID = 0, 1, 3

GEOMETRY_FLAG_DOUBLE_SIDED = 1 << 2
INSTANCE_FLAG_VISIBLE = 1 << 0
INSTANCE_FLAG_CASTS_SHADOW = 1 << 1
MATERIAL_FLAG_DOUBLE_SIDED = 1 << 0


class SceneDesc(C.Structure):
    _fields_ = [("triangles", C.c_void_p), ("triangle_count", C.c_uint32),
                ("nodes", C.c_void_p), ("node_count", C.c_uint32),
                ("build_kind", C.c_uint32), ("sah_bins", C.c_uint32), ("max_leaf_size", C.c_uint32),
                ("fingerprint", C.c_uint64), ("generation", C.c_uint32), ("device", C.c_uint32)]


class SceneInfo(C.Structure):
    _fields_ = [("triangle_count", C.c_uint32), ("node_count", C.c_uint32),
                ("max_depth", C.c_uint32), ("leaf_count", C.c_uint32),
                ("device_bytes", C.c_uint64), ("build_ms", C.c_double),
                ("node_bytes", C.c_uint32), ("triangle_bytes", C.c_uint32), ("gpu_build_ms", C.c_double)]


class TraceBatch(C.Structure):
    _fields_ = [("rays", C.c_void_p), ("hits", C.c_void_p), ("ray_offset", C.c_uint32),
                ("hit_offset", C.c_uint32), ("ray_count", C.c_uint32), ("memory", C.c_uint32),
                ("fingerprint", C.c_uint64), ("generation", C.c_uint32), ("reserved", C.c_uint32),
                ("stream", C.c_void_p)]


class TraversalCounters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "node_tests", "triangle_tests", "stack_overflows", "invalid_rays", "invalid_hits",
        "max_stack_depth", "leaf_visits", "leaf_primitives", "max_leaf_occupancy")]


class RendererDesc(C.Structure):
    _fields_ = [("max_width", C.c_uint32), ("max_height", C.c_uint32), ("max_depth", C.c_uint32),
                ("device", C.c_uint32)]


class RendererTuning(C.Structure):
    _fields_ = [("block_size", C.c_uint32), ("blocks_per_sm", C.c_uint32),
                ("fuse_intersect_shade", C.c_uint32), ("use_graph", C.c_uint32),
                ("shade_variant", C.c_uint32), ("traversal_refill", C.c_uint32),
                ("traversal_mode", C.c_uint32)]


class FrameTelemetry(C.Structure):
    _fields_ = [("path_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("fatal_mask", C.c_uint32),
                ("non_finite", C.c_uint32), ("negative_pdf", C.c_uint32), ("frames_accumulated", C.c_uint32),
                ("active_per_bounce", C.c_uint32 * 16), ("shadow_per_bounce", C.c_uint32 * 16),
                ("gpu_ms", C.c_double), ("total_path_rays", C.c_uint64), ("total_shadow_rays", C.c_uint64)]


class StageProfile(C.Structure):
    _fields_ = [("raygen_ms", C.c_float), ("resolve_ms", C.c_float), ("intersect_ms", C.c_float * 16),
                ("shade_ms", C.c_float * 16), ("shadow_ms", C.c_float * 16), ("rays", C.c_uint32 * 16),
                ("shadows", C.c_uint32 * 16), ("intersect_node_tests", C.c_uint64 * 16),
                ("intersect_triangle_tests", C.c_uint64 * 16), ("shadow_node_tests", C.c_uint64 * 16),
                ("shadow_triangle_tests", C.c_uint64 * 16), ("restir_ms", C.c_float),
                ("intersect_node_bytes", C.c_uint64 * 16), ("shadow_node_bytes", C.c_uint64 * 16)]


class RestirConfig(C.Structure):
    _fields_ = [("candidates", C.c_uint32), ("spatial_neighbors", C.c_uint32), ("max_m", C.c_uint32),
                ("max_history_age", C.c_uint32), ("temporal", C.c_uint32), ("neighbor_mode", C.c_uint32),
                ("disk_radius", C.c_float), ("normal_cos", C.c_float), ("relative_depth", C.c_float),
                ("position_distance", C.c_float), ("estimator", C.c_uint32)]


class RestirStatistics(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in (
        "candidates_generated", "candidates_valid", "candidates_rejected", "m_clamped", "temporal_attempts",
        "temporal_accepted", "spatial_attempts", "spatial_accepted", "visibility_submitted",
        "visibility_evaluated", "visibility_visible", "visibility_duplicate")]


class ViewDesc(C.Structure):
    _fields_ = [("frame", C.c_void_p), ("scene_slot", C.c_uint32), ("path_offset", C.c_uint32),
                ("accumulate", C.c_uint32), ("reserved", C.c_uint32), ("view_key", C.c_uint64)]


MAX_SCENE_SLOTS, MAX_BATCH_VIEWS = 32, 256


class ServerDesc(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("path_capacity", C.c_uint32), ("max_depth", C.c_uint32),
                ("device", C.c_uint32), ("max_batch_views", C.c_uint32), ("build_kind", C.c_uint32),
                ("restir", C.c_uint32), ("restir_config", RestirConfig), ("launch_paths", C.c_uint32),
                ("backfill_window", C.c_uint32)]


class RenderRequest(C.Structure):
    _fields_ = [("scene_key", C.c_uint64), ("frame", C.c_uint8 * 304), ("spp", C.c_uint32),
                ("reserved", C.c_uint32), ("arrival_time", C.c_double)]


class RequestStatus(C.Structure):
    _fields_ = [("state", C.c_uint32), ("samples_done", C.c_uint32), ("error", C.c_uint32),
                ("reserved", C.c_uint32), ("arrival_time", C.c_double), ("admit_time", C.c_double),
                ("completion_time", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "failed", "launches", "samples", "path_rays",
                                          "shadow_rays", "scene_builds", "evictions", "resident_bytes",
                                          "budget_bytes")] + \
               [(n, C.c_double) for n in ("latency_p50", "latency_p99", "latency_mean", "first_arrival",
                                          "last_completion")] + [("backfilled", C.c_uint64)]


assert C.sizeof(ServerDesc) == 88 and C.sizeof(RenderRequest) == 328 and C.sizeof(RestirConfig) == 44
assert C.sizeof(RequestStatus) == 40 and C.sizeof(ServerStats) == 136
BACKFILL_DEFAULT = 0xFFFFFFFF
REQUEST_WAITING, REQUEST_RUNNING, REQUEST_DONE, REQUEST_FAILED = 0, 1, 2, 3
RESTIR_PUBLISHED, RESTIR_TEMPORAL, RESTIR_SURFACES, RESTIR_DIRECT, RESTIR_REASONS = 0, 1, 2, 3, 4
ESTIMATOR_RESTIR_PRIMARY = 3


class SvgfConfig(C.Structure):
    _fields_ = [("relative_depth_threshold", C.c_float), ("absolute_depth_threshold", C.c_float),
                ("normal_cosine_threshold", C.c_float), ("require_material_id", C.c_uint32),
                ("require_object_id", C.c_uint32), ("max_history_length", C.c_uint32),
                ("minimum_color_alpha", C.c_float), ("minimum_moments_alpha", C.c_float),
                ("short_history_length", C.c_uint32), ("spatial_radius", C.c_uint32),
                ("minimum_variance", C.c_float), ("atrous_iterations", C.c_uint32), ("phi_depth", C.c_float),
                ("phi_normal", C.c_float), ("phi_luminance", C.c_float), ("minimum_albedo", C.c_float),
                ("demodulate_specular", C.c_uint32)]


class SvgfFrameInputs(C.Structure):
    _fields_ = [("gbuffer", C.c_void_p), ("raw_signal", C.c_void_p), ("width", C.c_uint32),
                ("height", C.c_uint32), ("memory", C.c_uint32), ("reset_trigger", C.c_uint32),
                ("frame_index", C.c_uint64)]


# Every symbol include/re_b200.h declares, with its ctypes signature.
_SIGNATURES = {
    "re_last_error": (C.c_char_p, []),
    "re_abi_version": (C.c_uint32, []),
    "re_execution_architecture_token": (C.c_char_p, []),
    "re_capability_is_built": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_char_p)]),
    "re_scene_create": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(C.c_void_p)]),
    "re_scene_destroy": (C.c_int, [C.c_void_p]),
    "re_scene_info_get": (C.c_int, [C.c_void_p, C.POINTER(SceneInfo)]),
    "re_scene_export_flat": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32]),
    "re_sah_build_host": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                    C.POINTER(C.c_uint32), C.c_void_p, C.POINTER(C.c_uint32)]),
    "re_renderer_profile": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(StageProfile)]),
    "re_trace_closest": (C.c_int, [C.c_void_p, C.POINTER(TraceBatch)]),
    "re_trace_any": (C.c_int, [C.c_void_p, C.POINTER(TraceBatch)]),
    "re_trace_counted": (C.c_int, [C.c_void_p, C.POINTER(TraceBatch), C.c_uint32,
                                   C.POINTER(TraversalCounters)]),
    "re_renderer_create": (C.c_int, [C.POINTER(RendererDesc), C.POINTER(C.c_void_p)]),
    "re_renderer_destroy": (C.c_int, [C.c_void_p]),
    "re_renderer_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(RendererTuning)]),
    "re_renderer_set_scene": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                        C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "re_renderer_render": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "re_renderer_read_film": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]),
    "re_renderer_collect": (C.c_int, [C.c_void_p, C.POINTER(FrameTelemetry)]),
    "re_renderer_film_pointer": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "re_svgf_default_config": (C.c_int, [C.POINTER(SvgfConfig)]),
    "re_svgf_create": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(SvgfConfig), C.c_uint32,
                                 C.POINTER(C.c_void_p)]),
    "re_svgf_destroy": (C.c_int, [C.c_void_p]),
    "re_svgf_set_config": (C.c_int, [C.c_void_p, C.POINTER(SvgfConfig)]),
    "re_svgf_get_config": (C.c_int, [C.c_void_p, C.POINTER(SvgfConfig)]),
    "re_svgf_reset": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "re_svgf_process": (C.c_int, [C.c_void_p, C.POINTER(SvgfFrameInputs), C.c_void_p]),
    "re_svgf_read": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]),
    "re_svgf_plane_pointer": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "re_svgf_select_output": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                        C.c_void_p]),
    "re_image_rmse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_float), C.c_void_p]),
    "re_bsdf_probe": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p]),
    "re_scene_set_alpha_masks": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32,
                                           C.c_uint32, C.c_uint32]),
    "re_lbvh_build_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "re_restir_default_config": (C.c_int, [C.POINTER(RestirConfig)]),
    "re_renderer_set_restir": (C.c_int, [C.c_void_p, C.POINTER(RestirConfig)]),
    "re_renderer_restir_reset": (C.c_int, [C.c_void_p]),
    "re_renderer_restir_statistics": (C.c_int, [C.c_void_p, C.POINTER(RestirStatistics)]),
    "re_renderer_restir_pointer": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    "re_renderer_restir_read": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]),
    "re_renderer_bind_scene": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                         C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "re_renderer_unbind_scene": (C.c_int, [C.c_void_p, C.c_uint32]),
    "re_renderer_set_environment": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32]),
    "re_renderer_environment_tables": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                                 C.POINTER(C.c_double)]),
    "re_renderer_render_views": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "re_renderer_read_view": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                        C.c_void_p]),
    "re_renderer_read_view_async": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                              C.c_void_p]),
    "re_renderer_wait_reads": (C.c_int, [C.c_void_p]),
    "re_scene_create_from_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "re_scene_expand_canonical": (C.c_int, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                            C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                            C.POINTER(C.c_uint32), C.c_uint32, C.c_uint32, C.c_void_p]),
    "re_renderer_restir_debug": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32,
                                           C.c_void_p]),
    "re_image_hash_linear_rgb": (C.c_int, [C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64,
                                           C.POINTER(C.c_uint64)]),
    "re_image_write_exr": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64]),
    "re_renderer_release_view": (C.c_int, [C.c_void_p, C.c_uint64]),
    "re_renderer_path_capacity": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    "re_plan_launches": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                   C.POINTER(C.c_uint32)]),
    "re_camera_matrices": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "re_renderer_export_reconstruction": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "re_server_create": (C.c_int, [C.POINTER(ServerDesc), C.POINTER(C.c_void_p)]),
    "re_server_destroy": (C.c_int, [C.c_void_p]),
    "re_server_clock": (C.c_double, [C.c_void_p]),
    "re_server_register_scene": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                           C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "re_server_submit": (C.c_int, [C.c_void_p, C.POINTER(RenderRequest), C.POINTER(C.c_uint64)]),
    "re_server_pump": (C.c_int, [C.c_void_p, C.c_uint32, C.c_double, C.POINTER(C.c_uint32)]),
    "re_server_drain": (C.c_int, [C.c_void_p]),
    "re_server_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(RequestStatus)]),
    "re_server_read_result": (C.c_int, [C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32]),
    "re_server_release": (C.c_int, [C.c_void_p, C.c_uint64]),
    "re_server_stats_get": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the built library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m renderingengine_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def declared_symbols() -> list[str]:
    return list(_SIGNATURES)


class NativeError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def check(code: int) -> None:
    if code != SUCCESS:
        msg = load().re_last_error()
        raise NativeError(code, msg.decode() if msg else "")


def ptr(a: np.ndarray | None) -> int | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data
