"""ctypes mirror of include/psycles_cuda.h and the loader of the in-tree
libpsycles_cuda.so.  The library is the product path: there is no Python or
CPU fallback, and loading fails loudly when the extension is missing."""

from __future__ import annotations

import ctypes
import os
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
# PSYCLES_CUDA_LIB selects a variant build (python -m psycles_b200.build --out)
LIB_PATH = pathlib.Path(os.environ.get("PSYCLES_CUDA_LIB") or HERE / "libpsycles_cuda.so")

c_float_p = ctypes.POINTER(ctypes.c_float)
c_uint32_p = ctypes.POINTER(ctypes.c_uint32)

PSY_OK = 0
(PSY_ERROR_INVALID_ARGUMENT, PSY_ERROR_OUT_OF_MEMORY, PSY_ERROR_CUDA, PSY_ERROR_CANCELLED, PSY_ERROR_RANGE,
 PSY_ERROR_UNSUPPORTED, PSY_ERROR_STATE, PSY_ERROR_TIMEOUT) = range(1, 9)
STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "out of memory", 3: "cuda error", 4: "cancelled",
    5: "range", 6: "unsupported", 7: "state", 8: "timeout",
}

(CLOSURE_NULL, CLOSURE_DIFFUSE, CLOSURE_EMISSION, CLOSURE_TRANSPARENT, CLOSURE_ADD, CLOSURE_MIX, CLOSURE_GLOSSY,
 CLOSURE_GLASS, CLOSURE_REFRACTION) = range(9)
GLOSSY_GGX, GLOSSY_BECKMANN, GLOSSY_MULTI_GGX = 0, 1, 2
MATERIAL_NO_BUMP_MAP_CORRECTION = 1
LIGHT_POINT, LIGHT_SPOT, LIGHT_AREA, LIGHT_DISTANT = range(4)
LIGHT_FLAG_SPHERE, LIGHT_FLAG_NORMALIZE, LIGHT_FLAG_ELLIPSE, LIGHT_FLAG_USE_MIS = 1, 2, 4, 8
VIS_CAMERA, VIS_DIFFUSE, VIS_GLOSSY, VIS_TRANSMISSION, VIS_SHADOW, VIS_VOLUME = 1, 2, 4, 8, 16, 32
VIS_ALL = 63
EMISSION_NONE, EMISSION_AUTOMATIC, EMISSION_FRONT, EMISSION_BACK, EMISSION_FRONT_BACK = range(5)
PASS_COMBINED, PASS_NORMAL, PASS_ALBEDO = 0, 2, 4
PASS_DENOISING_NORMAL, PASS_DENOISING_ALBEDO, PASS_SAMPLE_COUNT = 18, 19, 20
FILTER_BOX, FILTER_GAUSSIAN, FILTER_BLACKMAN_HARRIS = 0, 1, 2
DIRECT_MIS, DIRECT_FORWARD, DIRECT_NEE = 0, 1, 2
TRACE_MAX_EVENTS = 16
# closure inputs (psy_closure_instruction colour / scalar / roughness)
INPUT_VALUE, INPUT_NONE = 0x80000000, 0xFFFFFFFF
# value operations (compiler::ValueOperation numbering) and blend modes
VALUE_TYPE_SCALAR, VALUE_TYPE_VECTOR = 0, 1
(VALUE_PARAMETER, VALUE_PASSTHROUGH, VALUE_SCALAR_TO_COLOR, VALUE_SCALAR_TO_BOOLEAN, VALUE_COLOR_TO_SCALAR,
 VALUE_VECTOR_TO_SCALAR, VALUE_ADD, VALUE_SUBTRACT, VALUE_MULTIPLY, VALUE_DIVIDE, VALUE_MINIMUM, VALUE_MAXIMUM,
 VALUE_POWER) = range(13)
VALUE_ABSOLUTE, VALUE_CLAMP01, VALUE_CLAMP_RANGE = 14, 15, 16
VALUE_MIX_FLOAT, VALUE_MIX_VECTOR, VALUE_MIX, VALUE_MULTIPLY_COLOR, VALUE_INVERT = 21, 22, 23, 24, 26
VALUE_SEPARATE_R, VALUE_SEPARATE_G, VALUE_SEPARATE_B, VALUE_COMBINE_COLOR = 100, 101, 102, 103
BLEND_MIX, BLEND_DARKEN, BLEND_MULTIPLY, BLEND_LIGHTEN, BLEND_SCREEN, BLEND_ADD = 0, 1, 2, 4, 5, 7
BLEND_DIFFERENCE, BLEND_SUBTRACT = 11, 13


class MeshDesc(ctypes.Structure):
    _fields_ = [("positions", c_float_p), ("normals", c_float_p), ("indices", c_uint32_p),
                ("materials", c_uint32_p), ("vertex_count", ctypes.c_uint32),
                ("triangle_count", ctypes.c_uint32), ("smooth", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class InstanceDesc(ctypes.Structure):
    _fields_ = [("object_to_world", ctypes.c_float * 16), ("mesh", ctypes.c_uint32),
                ("material", ctypes.c_uint32), ("visibility", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ClosureInstruction(ctypes.Structure):
    _fields_ = [("op", ctypes.c_uint32), ("a", ctypes.c_uint32), ("b", ctypes.c_uint32),
                ("color", ctypes.c_uint32), ("scalar", ctypes.c_uint32), ("roughness", ctypes.c_uint32)]


class ValueInstruction(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("op", "type", "parameter", "a", "b", "c", "static_u0", "static_u1")]


class MaterialDesc(ctypes.Structure):
    _fields_ = [("closures", ctypes.POINTER(ClosureInstruction)), ("closure_count", ctypes.c_uint32),
                ("root", ctypes.c_uint32), ("scalars", c_float_p), ("scalar_count", ctypes.c_uint32),
                ("vector_count", ctypes.c_uint32), ("vectors", c_float_p),
                ("emission_sampling", ctypes.c_uint32), ("value_count", ctypes.c_uint32),
                ("values", ctypes.POINTER(ValueInstruction)), ("flags", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class LightDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("max_bounces", ctypes.c_uint32),
                ("visibility", ctypes.c_uint32), ("position", ctypes.c_float * 3), ("axis_x", ctypes.c_float * 3),
                ("axis_y", ctypes.c_float * 3), ("axis_z", ctypes.c_float * 3), ("axis_scale", ctypes.c_float * 3),
                ("color", ctypes.c_float * 3), ("power", ctypes.c_float), ("radius", ctypes.c_float),
                ("size_u", ctypes.c_float), ("size_v", ctypes.c_float), ("spot_angle", ctypes.c_float),
                ("spot_smooth", ctypes.c_float), ("angle", ctypes.c_float), ("spread", ctypes.c_float)]


class CameraDesc(ctypes.Structure):
    _fields_ = [("camera_to_world", ctypes.c_float * 16), ("field_of_view", ctypes.c_float),
                ("horizontal_field_of_view", ctypes.c_float), ("sensor_fit", ctypes.c_uint32),
                ("lens_shift_x", ctypes.c_float), ("lens_shift_y", ctypes.c_float),
                ("near_clip", ctypes.c_float), ("far_clip", ctypes.c_float), ("projection", ctypes.c_uint32),
                ("orthographic_scale", ctypes.c_float), ("aperture_radius", ctypes.c_float),
                ("focal_distance", ctypes.c_float), ("aperture_blades", ctypes.c_uint32),
                ("aperture_rotation", ctypes.c_float), ("aperture_ratio", ctypes.c_float),
                ("reserved", ctypes.c_uint32)]


CAMERA_PERSPECTIVE, CAMERA_ORTHOGRAPHIC, CAMERA_PANORAMA = 0, 1, 2


class SceneDesc(ctypes.Structure):
    _fields_ = [("meshes", ctypes.POINTER(MeshDesc)), ("instances", ctypes.POINTER(InstanceDesc)),
                ("materials", ctypes.POINTER(MaterialDesc)), ("lights", ctypes.POINTER(LightDesc)),
                ("mesh_count", ctypes.c_uint32), ("instance_count", ctypes.c_uint32),
                ("material_count", ctypes.c_uint32), ("light_count", ctypes.c_uint32),
                ("camera", CameraDesc), ("background", ctypes.c_float * 3),
                ("world_visibility", ctypes.c_uint32), ("revision", ctypes.c_uint64),
                ("ggx_e", c_float_p), ("ggx_eavg", c_float_p)]


class RenderSettings(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "full_width", "full_height", "window_x", "window_y", "window_width", "window_height", "seed",
        "transparent_background", "pixel_filter")] + [
        ("filter_width", ctypes.c_float), ("pass_alpha_threshold", ctypes.c_float)] + [
        (n, ctypes.c_uint32) for n in (
            "max_bounces", "min_bounces", "diffuse_bounces", "glossy_bounces", "transmission_bounces",
            "transparent_min_bounces", "transparent_max_bounces")] + [
        (n, ctypes.c_float) for n in (
            "sample_clamp_direct", "sample_clamp_indirect", "film_exposure", "light_sampling_threshold")] + [
        (n, ctypes.c_uint32) for n in (
            "use_light_tree", "direct_light_sampling", "next_event_estimation", "reserved")]


class PathEvent(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "rng_offset", "bounce", "transparent_bounce", "flag", "visibility", "hit_object", "hit_primitive",
        "closure_index", "label", "light_kind", "light_index", "terminated")] + [
        ("hit_t", ctypes.c_float), ("hit_u", ctypes.c_float), ("hit_v", ctypes.c_float),
        ("random_terminate", ctypes.c_float), ("random_light", ctypes.c_float * 3),
        ("random_light_terminate", ctypes.c_float), ("random_bsdf", ctypes.c_float * 3),
        ("continuation_probability", ctypes.c_float), ("bsdf_pdf", ctypes.c_float),
        ("wi", ctypes.c_float * 3), ("throughput", ctypes.c_float * 3), ("emission", ctypes.c_float * 3),
        ("nee", ctypes.c_float * 3)]


class PathTrace(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in (
        "pixel_x", "pixel_y", "sample", "rng_hash", "event_count", "valid")] + [
        ("filter", ctypes.c_float * 2), ("ray_origin", ctypes.c_float * 3),
        ("ray_direction", ctypes.c_float * 3), ("radiance", ctypes.c_float * 3),
        ("events", PathEvent * TRACE_MAX_EVENTS)]


class RenderStats(ctypes.Structure):
    _fields_ = [("camera_rays", ctypes.c_uint64), ("closest_rays", ctypes.c_uint64),
                ("shadow_rays", ctypes.c_uint64), ("path_segments", ctypes.c_uint64),
                ("ms_total", ctypes.c_float), ("ms_intersect", ctypes.c_float), ("ms_shade", ctypes.c_float),
                ("ms_shadow", ctypes.c_float), ("ms_film", ctypes.c_float),
                ("kernel_launches", ctypes.c_uint32), ("batches", ctypes.c_uint32)]


class KernelProfile(ctypes.Structure):
    _fields_ = [(n + "_launches", ctypes.c_uint32) for n in ("raygen", "intersect", "shade", "shadow", "film")] + [
        ("reserved", ctypes.c_uint32)] + [
        (n + "_ms", ctypes.c_float) for n in ("raygen", "intersect", "shade", "shadow", "film")] + [
        ("reserved_ms", ctypes.c_float)] + [
        (n + "_bytes", ctypes.c_double) for n in ("raygen", "intersect", "shade", "shadow", "film")] + [
        ("reserved_bytes", ctypes.c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint32) for n in ("path_capacity", "stream_blocks_per_sm", "traversal_blocks_per_sm",
                                               "shade_blocks_per_sm", "sort_threshold", "shadow_sort_threshold",
                                               "ray_sort_threshold", "stream_block_size")]


class BatchConfig(ctypes.Structure):
    _fields_ = [("path_capacity", ctypes.c_uint32), ("max_jobs", ctypes.c_uint32), ("use_graph", ctypes.c_uint32),
                ("check_interval", ctypes.c_uint32)]


class BatchStats(ctypes.Structure):
    _fields_ = [("samples", ctypes.c_uint64), ("closest_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
                ("ms_total", ctypes.c_float), ("wavefronts", ctypes.c_uint32), ("jobs", ctypes.c_uint32),
                ("graph_launches", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("path_capacity", ctypes.c_uint32),
                ("max_running", ctypes.c_uint32), ("use_graph", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class JobInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_uint32), ("status", ctypes.c_int32), ("samples_done", ctypes.c_uint32),
                ("samples_total", ctypes.c_uint32), ("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double),
                ("done_ms", ctypes.c_double)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("jobs_submitted", "jobs_done", "jobs_failed", "samples", "wavefronts",
                                               "bytes_in_use", "bytes_peak")] + [
        ("busy_ms", ctypes.c_double), ("latency_p50_ms", ctypes.c_double), ("latency_p99_ms", ctypes.c_double),
        ("latency_jobs", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("device_ms", ctypes.c_double)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = 0, 1, 2, 3, 4


class SceneBuildStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("total_ms", "validate_ms", "blas_ms", "tlas_ms", "emitters_ms",
                                               "upload_ms", "light_tree_ms")] + [
        ("build_threads", ctypes.c_uint32), ("light_tree_builds", ctypes.c_uint32),
        ("stack_need", ctypes.c_uint32), ("stack_capacity", ctypes.c_uint32), ("median_rebuilds", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32), ("upload_bytes", ctypes.c_uint64)]


# Entry points declared by include/psycles_cuda.h: (name, restype, argtypes).
SIGNATURES = [
    ("psy_last_error", ctypes.c_char_p, []),
    ("psy_abi_version", ctypes.c_uint32, []),
    ("psy_render_settings_default", None, [ctypes.POINTER(RenderSettings)]),
    ("psy_context_create", ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("psy_context_destroy", None, [ctypes.c_void_p]),
    ("psy_scene_compile", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SceneDesc), ctypes.POINTER(ctypes.c_void_p)]),
    ("psy_scene_destroy", None, [ctypes.c_void_p]),
    ("psy_scene_source_revision", ctypes.c_uint64, [ctypes.c_void_p]),
    ("psy_scene_get_build_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SceneBuildStats)]),
    ("psy_scene_rebind_parameters", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, c_float_p, ctypes.c_uint32, c_float_p, ctypes.c_uint32]),
    ("psy_session_create", ctypes.c_int,
     [ctypes.c_void_p, ctypes.POINTER(RenderSettings), ctypes.POINTER(ctypes.c_void_p)]),
    ("psy_session_destroy", None, [ctypes.c_void_p]),
    ("psy_session_reset", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RenderSettings)]),
    ("psy_session_render_samples", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("psy_session_render_samples_static", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("psy_session_cancel", None, [ctypes.c_void_p]),
    ("psy_session_read_pass", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, c_float_p, ctypes.c_uint64, c_uint32_p]),
    ("psy_session_rendered_samples", ctypes.c_uint32, [ctypes.c_void_p]),
    ("psy_session_request_trace", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]),
    ("psy_session_read_trace", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PathTrace)]),
    ("psy_session_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(RenderStats)]),
    ("psy_session_set_profiling", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32]),
    ("psy_session_profile", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(KernelProfile)]),
    ("psy_sobol_sequence_size_for_samples", ctypes.c_uint32, [ctypes.c_uint32]),
    ("psy_sobol_generate_table", ctypes.c_int, [ctypes.c_uint32, c_float_p]),
    ("psy_pixel_filter_table", ctypes.c_int, [ctypes.c_uint32, ctypes.c_float, c_float_p]),
    ("psy_debug_sobol_samples", ctypes.c_int,
     [ctypes.c_void_p, ctypes.c_uint32, c_uint32_p, ctypes.c_uint32, c_float_p, c_uint32_p]),
    ("psy_session_set_camera", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("psy_context_set_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    ("psy_context_get_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Tuning)]),
    ("psy_batch_create", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchConfig), ctypes.POINTER(ctypes.c_void_p)]),
    ("psy_batch_destroy", None, [ctypes.c_void_p]),
    ("psy_batch_render", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), c_uint32_p, c_uint32_p,
                                        c_uint32_p, c_uint32_p, ctypes.c_uint32]),
    ("psy_batch_get_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(BatchStats)]),
    ("psy_batch_plan", ctypes.c_int, [c_uint32_p, c_uint32_p, ctypes.c_uint32, ctypes.c_uint32, c_uint32_p,
                                      ctypes.c_uint32, c_uint32_p]),
    ("psy_server_create", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerConfig),
                                         ctypes.POINTER(ctypes.c_void_p)]),
    ("psy_server_destroy", None, [ctypes.c_void_p]),
    ("psy_server_submit", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]),
    ("psy_server_rebind_parameters", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, c_float_p,
                                                    ctypes.c_uint32, c_float_p, ctypes.c_uint32]),
    ("psy_server_poll", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(JobInfo)]),
    ("psy_server_wait", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32]),
    ("psy_server_read_pass", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, c_float_p,
                                            ctypes.c_uint64, c_uint32_p]),
    ("psy_server_release", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("psy_server_cancel", ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    ("psy_server_get_stats", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    ("psy_scene_device_bytes", ctypes.c_uint64, [ctypes.c_void_p]),
    ("psy_debug_light_tree", ctypes.c_int,
     [ctypes.c_void_p, c_float_p, c_uint32_p, ctypes.c_uint32, c_uint32_p, c_float_p, c_float_p]),
    ("psy_debug_light_distribution", ctypes.c_int,
     [ctypes.c_void_p, c_float_p, ctypes.c_uint32, c_uint32_p, c_uint32_p, c_float_p]),
]

def default_settings() -> RenderSettings:
    """contract::RenderSettings / PathIntegratorSettings defaults
    (include/psycles/contract/render.h:81-115); equals psy_render_settings_default."""
    s = RenderSettings()
    s.filter_width = 1.0
    s.pass_alpha_threshold = 0.5
    s.max_bounces, s.diffuse_bounces, s.glossy_bounces = 12, 4, 4
    s.transmission_bounces, s.transparent_max_bounces = 12, 8
    s.film_exposure = 1.0
    s.light_sampling_threshold = 0.01
    s.direct_light_sampling = DIRECT_MIS
    s.next_event_estimation = 1
    return s


_lib = None


class PsyError(RuntimeError):
    """A psy_status other than PSY_OK, with psy_last_error()'s message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load() -> ctypes.CDLL:
    """Loads the in-tree libpsycles_cuda.so (built by psycles_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m psycles_b200.build` first")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, restype, argtypes in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != PSY_OK:
        raise PsyError(status, load().psy_last_error().decode())


def ptr(array, ctype=ctypes.c_float):
    """Pointer to a contiguous numpy array (or None for None)."""
    if array is None:
        return ctypes.cast(None, ctypes.POINTER(ctype))
    return array.ctypes.data_as(ctypes.POINTER(ctype))
