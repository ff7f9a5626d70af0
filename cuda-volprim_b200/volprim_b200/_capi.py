"""ctypes bindings of libvolprim_b200.so (declarations in include/volprim_b200.h).

The library is the only compute path: if it is missing or fails to load, importing this module
raises, naming the build step (cuda-volprim_b200/build_lib.py or __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libvolprim_b200.so"

VP_OK = 0
VP_MEMORY_HOST, VP_MEMORY_DEVICE = 0, 1
VP_NEE_MIS, VP_NEE_PHASE, VP_NEE_RIS, VP_NEE_NONE = 0, 1, 2, 3
VP_ENGINE_WARP, VP_ENGINE_MEGAKERNEL, VP_ENGINE_WAVEFRONT = 0, 1, 2
VP_PRECISION_AUTO, VP_PRECISION_FAST, VP_PRECISION_ACCURATE = 0, 1, 2
VP_MEASURE_COUNTERS, VP_MEASURE_STAGES = 1, 2
VP_SCHEDULE_FIFO, VP_SCHEDULE_FAIR, VP_SCHEDULE_SRPT = 0, 1, 2
VP_TREE_PLOC, VP_TREE_LBVH = 0, 1
VP_COLLAPSE_GREEDY, VP_COLLAPSE_SAH = 0, 1
VP_TAU_ORDER_AUTO, VP_TAU_ORDER_LANE, VP_TAU_ORDER_NEAREST = 0, 1, 2

ERROR_NAMES = {
    -1: "VP_ERROR_INVALID_ARGUMENT", -2: "VP_ERROR_CUDA", -3: "VP_ERROR_OUT_OF_MEMORY",
    -4: "VP_ERROR_UNSUPPORTED", -5: "VP_ERROR_LIMIT", -6: "VP_ERROR_DEVICE_STATUS",
    -7: "VP_ERROR_INTERNAL",
}


class VpError(RuntimeError):
    """A vp_* call returned a negative vp_status."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{ERROR_NAMES.get(status, status)}: {message}")


class vp_gaussians(C.Structure):
    _fields_ = [
        ("count", C.c_uint32),
        ("mean", C.c_void_p),
        ("scale", C.c_void_p),
        ("quat_wxyz", C.c_void_p),
        ("density", C.c_void_p),
        ("albedo", C.c_void_p),
        ("scale_is_log", C.c_int32),
        ("memory", C.c_int32),
    ]


class vp_scene_info(C.Structure):
    _fields_ = [
        ("count", C.c_uint32),
        ("wide_nodes", C.c_uint32),
        ("wide_depth", C.c_uint32),
        ("binary_nodes", C.c_uint32),
        ("leaves", C.c_uint32),
        ("albedo_all_zero", C.c_int32),
        ("build_ms", C.c_double),
        ("bounds_min", C.c_double * 3),
        ("bounds_max", C.c_double * 3),
        ("device_bytes", C.c_uint64),
        ("wide_builder", C.c_int32),
        ("binary_builder", C.c_int32),
        ("binary_height", C.c_uint32),
        ("leaf_max", C.c_uint32),
        ("wide_collapse", C.c_int32),
        ("tau_order", C.c_int32),
    ]


class vp_scene_options(C.Structure):
    _fields_ = [
        ("wide_builder", C.c_int32),
        ("binary_builder", C.c_int32),
        ("leaf_max", C.c_uint32),
        ("wide_collapse", C.c_int32),
        ("tau_order", C.c_int32),
    ]


class vp_camera(C.Structure):
    _fields_ = [
        ("eye", C.c_float * 3),
        ("lookat", C.c_float * 3),
        ("up", C.c_float * 3),
        ("vfov_deg", C.c_float),
        ("ortho_height", C.c_float),
        ("orthographic", C.c_int32),
    ]


class vp_render_params(C.Structure):
    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("spp", C.c_uint32),
        ("seed", C.c_uint32),
        ("max_bounces", C.c_uint32),
        ("rr_depth", C.c_uint32),
        ("rr_max_survival", C.c_float),
        ("hg_g", C.c_float),
        ("firefly_clamp", C.c_float),
        ("pixel_filter_stddev", C.c_float),
        ("nee_mode", C.c_int32),
        ("ris_candidates", C.c_uint32),
        ("batch_spp", C.c_uint32),
        ("engine", C.c_int32),
        ("precision", C.c_int32),
        ("measure", C.c_int32),
        ("adaptive_threshold", C.c_float),
        ("adaptive_min_samples", C.c_uint32),
    ]


class vp_render_stats(C.Structure):
    _fields_ = [
        ("ms_kernels", C.c_double),
        ("paths", C.c_uint64),
        ("bounces", C.c_uint64),
        ("scatters", C.c_uint64),
        ("crossings", C.c_uint64),
        ("shadow_rays", C.c_uint64),
        ("nodes_visited", C.c_uint64),
        ("leaves_visited", C.c_uint64),
        ("prim_tests", C.c_uint64),
        ("geo_loads", C.c_uint64),
        ("query_nodes", C.c_uint64 * 3),
        ("query_leaves", C.c_uint64 * 3),
        ("max_hits_per_ray", C.c_uint32),
        ("max_point_overlap", C.c_uint32),
        ("device_status", C.c_uint32),
        ("launches", C.c_uint32),
        ("query_prim_tests", C.c_uint64 * 3),
        ("query_geo_loads", C.c_uint64 * 3),
        ("ms_stage", C.c_double * 3),
        ("stage_launches", C.c_uint32 * 3),
        ("reserved", C.c_uint32),
        ("paths_skipped", C.c_uint64),
        ("hits_hist", (C.c_uint64 * 16) * 2),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            if name == "reserved":
                continue
            v = getattr(self, name)
            if isinstance(v, C.Array):
                v = [list(x) if isinstance(x, C.Array) else x for x in v]
            out[name] = v
        return out


class vp_gaussian_grads(C.Structure):
    _fields_ = [
        ("mean", C.c_void_p),
        ("scale", C.c_void_p),
        ("quat_wxyz", C.c_void_p),
        ("density", C.c_void_p),
        ("emission", C.c_void_p),
        ("memory", C.c_int32),
    ]


class vp_host_gaussians(C.Structure):
    _fields_ = [
        ("count", C.c_uint32),
        ("mean", C.POINTER(C.c_float)),
        ("log_scale", C.POINTER(C.c_float)),
        ("quat_wxyz", C.POINTER(C.c_float)),
        ("density", C.POINTER(C.c_float)),
        ("albedo", C.POINTER(C.c_float)),
    ]


class vp_server_config(C.Structure):
    _fields_ = [
        ("memory_budget_bytes", C.c_uint64),
        ("path_slots", C.c_uint32),
        ("max_requests", C.c_uint32),
        ("iterations_per_step", C.c_uint32),
        ("precision", C.c_int32),
        ("use_graph", C.c_int32),
        ("schedule", C.c_int32),
        ("srpt_reserve", C.c_float),
        ("lanes", C.c_uint32),
        ("srpt_aging", C.c_float),
    ]


class vp_request(C.Structure):
    _fields_ = [
        ("scene_id", C.c_uint32),
        ("camera", vp_camera),
        ("params", vp_render_params),
        ("out_rgba", C.c_void_p),
        ("memory", C.c_int32),
        ("reserved", C.c_int32),
    ]


class vp_server_stats(C.Structure):
    _fields_ = [
        ("submitted", C.c_uint64),
        ("admitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("paths_completed", C.c_uint64),
        ("iterations", C.c_uint64),
        ("active", C.c_uint32),
        ("pending", C.c_uint32),
        ("bytes_in_use", C.c_uint64),
        ("device_ms", C.c_double),
        ("cancelled", C.c_uint64),
        ("alloc_failures", C.c_uint64),
    ]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)

# name -> argtypes (every function returns vp_status unless listed in _RESTYPES)
SIGNATURES = {
    "vp_last_error_string": [],
    "vp_version": [C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
    "vp_context_create": [C.c_int32, PP],
    "vp_context_destroy": [P],
    "vp_context_stream": [P, PP],
    "vp_context_synchronize": [P],
    "vp_context_sm_count": [P, C.POINTER(C.c_int32)],
    "vp_scene_create": [P, C.POINTER(vp_gaussians), C.c_float, PP],
    "vp_scene_options_default": [C.POINTER(vp_scene_options)],
    "vp_scene_create_ex": [P, C.POINTER(vp_gaussians), C.c_float, C.POINTER(vp_scene_options), PP],
    "vp_scene_info_get": [P, C.POINTER(vp_scene_info)],
    "vp_scene_destroy": [P],
    "vp_env_create": [P, P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int32, PP],
    "vp_env_create_constant": [P, C.c_float, C.c_float, C.c_float, PP],
    "vp_env_build_ms": [P, C.POINTER(C.c_double)],
    "vp_env_read_tables": [P, P, P, P, P, P, P, P, P],
    "vp_env_destroy": [P],
    "vp_render_params_default": [C.POINTER(vp_render_params)],
    "vp_image_create": [P, C.c_uint32, C.c_uint32, PP],
    "vp_image_clear": [P],
    "vp_image_destroy": [P],
    "vp_image_read": [P, P, C.c_int32],
    "vp_image_device_buffers": [P, PP, PP],
    "vp_image_read_welford": [P, P, P, C.c_int32],
    "vp_render_accumulate": [P, P, C.POINTER(vp_camera), C.POINTER(vp_render_params), P, C.c_uint32,
                             C.c_uint32, C.POINTER(vp_render_stats)],
    "vp_render": [P, P, C.POINTER(vp_camera), C.POINTER(vp_render_params), P, C.c_int32,
                  C.POINTER(vp_render_stats)],
    "vp_transmittance": [P, P, P, C.c_uint32, C.c_int32, C.c_int32, P, C.c_int32],
    "vp_albedo_at": [P, P, C.c_uint32, C.c_int32, C.c_int32, P, P, C.c_int32],
    "vp_transmittance_static": [P, P, P, C.c_uint32, C.c_int32, P, C.c_int32],
    "vp_camera_rays": [P, C.POINTER(vp_camera), C.POINTER(vp_render_params), P, P, P, C.c_uint32, P, P, C.c_int32],
    "vp_normalize_accumulator": [P, P, P, C.c_size_t, C.c_float, P],
    "vp_scene_set_emission": [P, P, C.c_int32],
    "vp_render_emission": [P, P, C.POINTER(vp_camera), C.POINTER(vp_render_params), P, C.c_int32,
                           C.POINTER(vp_render_stats)],
    "vp_render_emission_backward": [P, P, C.POINTER(vp_camera), C.POINTER(vp_render_params), P, C.c_int32,
                                    C.POINTER(vp_gaussian_grads), C.POINTER(vp_render_stats)],
    "vp_server_create": [P, C.POINTER(vp_server_config), PP],
    "vp_server_add_scene": [P, P, P, C.POINTER(C.c_uint32)],
    "vp_server_submit": [P, C.POINTER(vp_request), C.POINTER(C.c_uint64)],
    "vp_server_step": [P, C.POINTER(C.c_uint32)],
    "vp_server_cancel": [P, C.c_uint64],
    "vp_server_inject_alloc_failures": [P, C.c_uint32],
    "vp_server_poll": [P, C.POINTER(C.c_uint64), C.c_uint32, C.POINTER(C.c_uint32)],
    "vp_server_get_stats": [P, C.POINTER(vp_server_stats)],
    "vp_server_destroy": [P],
    "vp_ply_load": [C.c_char_p, P, C.POINTER(vp_host_gaussians)],
    "vp_ply_save": [C.c_char_p, C.POINTER(vp_host_gaussians)],
    "vp_host_gaussians_free": [C.POINTER(vp_host_gaussians)],
    "vp_hdr_load": [C.c_char_p, C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
    "vp_host_free": [P],
    "vp_exr_save": [C.c_char_p, P, C.c_uint32, C.c_uint32, C.c_int32],
}
_RESTYPES = {"vp_last_error_string": C.c_char_p}


def load_library(path: Path | str | None = None) -> C.CDLL:
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python cuda-volprim_b200/build_lib.py` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = C.CDLL(str(p))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = _RESTYPES.get(name, C.c_int32)
    return lib


lib = load_library()


def check(status: int) -> None:
    if status != VP_OK:
        msg = lib.vp_last_error_string()
        raise VpError(status, msg.decode() if msg else "")
