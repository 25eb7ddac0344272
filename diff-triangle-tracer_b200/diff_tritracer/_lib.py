"""ctypes binding of libtritracer.so, the C ABI declared in include/tritracer.h.

The library is built in-tree (``make -C diff-triangle-tracer_b200``). There is
no fallback: importing this module without the built library raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# TRITRACER_LIB selects another build of the library, e.g. the index-checked
# libtritracer_bounds.so (`make bounds`)
LIB_PATH = os.environ.get("TRITRACER_LIB") or os.path.join(_HERE, "libtritracer.so")

TT_OK = 0
TT_ERR_INVALID = 1
TT_ERR_OOM = 2
TT_ERR_TIMEOUT = 3
TT_ERR_STACK = 4
TT_ERR_CUDA = 5
TT_ERR_STATE = 6

TT_VARIANT_PLAIN = 0
TT_VARIANT_REFLECT = 1
TT_VARIANT_REFRACT = 2
TT_VARIANT_ENVLIGHT = 3

TT_OPT_SPLIT_FORWARD = 1
TT_OPT_SORT_SECONDARY = 2
TT_OPT_COLLECT_QUERIES = 3
TT_OPT_WORK_COUNTERS = 4

TT_TRAVERSAL_AUTO = 0
TT_TRAVERSAL_PACKETS = 1
TT_TRAVERSAL_LANES = 2

_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


class TtConfig(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int), ("tmin_inclusive", ctypes.c_int), ("traversal", ctypes.c_int),
                ("k", ctypes.c_int), ("stack_depth", ctypes.c_int), ("exact_adjoint", ctypes.c_int),
                ("reference_arithmetic", ctypes.c_int), ("reserved", ctypes.c_int * 1)]


class TtFwdArgs(ctypes.Structure):
    _fields_ = [
        ("H", ctypes.c_int), ("W", ctypes.c_int),
        ("ray_o", _vp), ("ray_d", _vp),
        ("vertices", _vp), ("num_vertices", ctypes.c_int),
        ("num_points", _vp), ("cumsum", _vp), ("P", ctypes.c_int),
        ("shs", _vp), ("sh_degree", ctypes.c_int), ("M", ctypes.c_int),
        ("colors_precomp", _vp), ("opacities", _vp), ("sigma", _vp),
        ("scaling", _vp), ("density_factor", _vp),
        ("bg", _vp), ("extra", _vp), ("extra_len", ctypes.c_int),
        ("rebuild_gas", ctypes.c_int), ("debug", ctypes.c_int),
        ("out_color", _vp), ("out_others", _vp), ("max_blending", _vp),
        ("gpu_time_ms", _f),
        ("hit_cache", _vp), ("hit_cache_bytes", ctypes.c_size_t),
    ]


class TtBwdArgs(ctypes.Structure):
    _fields_ = [
        ("H", ctypes.c_int), ("W", ctypes.c_int),
        ("ray_o", _vp), ("ray_d", _vp), ("bg", _vp),
        ("vertices", _vp), ("num_vertices", ctypes.c_int),
        ("sigma", _vp), ("num_points", _vp), ("cumsum", _vp),
        ("colors", _vp), ("others", _vp), ("P", ctypes.c_int),
        ("shs", _vp), ("sh_degree", ctypes.c_int), ("M", ctypes.c_int),
        ("opacities", _vp), ("dL_dpixels", _vp), ("dL_dothers", _vp), ("scaling", _vp),
        ("debug", ctypes.c_int),
        ("dL_dtriangle", _vp), ("dL_dsigma", _vp), ("dL_dopacity", _vp), ("dL_dsh", _vp),
        ("gpu_time_ms", _f),
        ("colors_precomp", _vp), ("dL_dcolors", _vp),
        ("hit_cache", _vp), ("hit_cache_bytes", ctypes.c_size_t),
    ]


class TtView(ctypes.Structure):
    _fields_ = [("H", ctypes.c_int), ("W", ctypes.c_int), ("ray_o", _vp), ("ray_d", _vp),
                ("out_color", _vp), ("out_others", _vp), ("colors", _vp), ("others", _vp),
                ("dL_dpixels", _vp), ("dL_dothers", _vp), ("interval", _vp), ("record", _vp)]


class TtCamera(ctypes.Structure):
    _fields_ = [("origin", ctypes.c_double * 3), ("forward", ctypes.c_double * 3), ("right", ctypes.c_double * 3),
                ("up", ctypes.c_double * 3), ("tan_half_fov", ctypes.c_double), ("H", ctypes.c_int),
                ("W", ctypes.c_int), ("ray_o", _vp), ("ray_d", _vp)]


class TtStats(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_ulonglong), ("evaluated_hits", ctypes.c_ulonglong),
                ("blended_hits", ctypes.c_ulonglong), ("kernel_launches", ctypes.c_ulonglong),
                ("node_visits", ctypes.c_ulonglong), ("triangle_tests", ctypes.c_ulonglong),
                ("queries", ctypes.c_ulonglong), ("packet_node_visits", ctypes.c_ulonglong),
                ("interval_continuations", ctypes.c_ulonglong), ("interval_retraces", ctypes.c_ulonglong),
                ("hit_cache_replays", ctypes.c_ulonglong)]


TT_MLP_PARAMS = 16640
TT_MLP_PARTIAL = 16656


class TtMlp(ctypes.Structure):
    _fields_ = [("weights", _vp), ("master", _vp), ("adam_m", _vp), ("adam_v", _vp), ("partial", _vp),
                ("partial_ctas", ctypes.c_int), ("origin_scale", ctypes.c_float), ("t_shift", ctypes.c_float),
                ("t_scale", ctypes.c_float), ("center", ctypes.c_float * 3)]


class TtMlpStep(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("step", ctypes.c_int), ("near_weight", ctypes.c_float),
                ("far_weight", ctypes.c_float)]


class TtSecondary(ctypes.Structure):
    _fields_ = [("material", _vp), ("ior", _vp), ("env", _vp), ("env_h", ctypes.c_int), ("env_w", ctypes.c_int),
                ("max_depth", ctypes.c_int), ("dL_denv", _vp), ("dL_dior", _vp)]


EXPORTS = (
    "tt_create", "tt_destroy", "tt_build", "tt_forward", "tt_backward", "tt_last_error",
    "tt_device_status", "tt_hit_stream", "tt_get_stats", "tt_reset_stats", "tt_forward_views",
    "tt_backward_views", "tt_set_traversal", "tt_set_option", "tt_forward_pass_times", "tt_mlp_update",
    "tt_mlp_train_step", "tt_mlp_predict",
    "tt_mlp_intervals", "tt_forward_secondary", "tt_backward_secondary", "tt_secondary_tree", "tt_bvh_save",
    "tt_bvh_load", "tt_hit_cache_bytes", "tt_hit_cache_bytes_pool", "tt_hit_cache_usage",
    "tt_camera_rays",
)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"diff_tritracer: {LIB_PATH} is missing; build it with `make -C {os.path.dirname(_HERE)}` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.tt_create.argtypes = [ctypes.POINTER(TtConfig), ctypes.POINTER(_vp)]
    lib.tt_destroy.argtypes = [_vp]
    lib.tt_build.argtypes = [_vp, _vp, ctypes.c_int, _vp, ctypes.c_int, ctypes.c_int, _vp]
    lib.tt_forward.argtypes = [_vp, ctypes.POINTER(TtFwdArgs), _vp]
    lib.tt_backward.argtypes = [_vp, ctypes.POINTER(TtBwdArgs), _vp]
    lib.tt_last_error.argtypes = [_vp]
    lib.tt_last_error.restype = ctypes.c_char_p
    lib.tt_device_status.argtypes = [_vp, _vp]
    lib.tt_forward_views.argtypes = [_vp, ctypes.POINTER(TtFwdArgs), ctypes.POINTER(TtView), ctypes.c_int, _vp]
    lib.tt_backward_views.argtypes = [_vp, ctypes.POINTER(TtBwdArgs), ctypes.POINTER(TtView), ctypes.c_int, _vp]
    lib.tt_set_traversal.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.tt_set_option.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    lib.tt_forward_pass_times.argtypes = [_vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    lib.tt_get_stats.argtypes = [_vp, ctypes.POINTER(TtStats), _vp]
    lib.tt_reset_stats.argtypes = [_vp, _vp]
    lib.tt_hit_stream.argtypes = [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]
    lib.tt_forward_secondary.argtypes = [_vp, ctypes.POINTER(TtFwdArgs), ctypes.POINTER(TtSecondary), _vp]
    lib.tt_backward_secondary.argtypes = [_vp, ctypes.POINTER(TtBwdArgs), ctypes.POINTER(TtSecondary), _vp]
    lib.tt_bvh_save.argtypes = [_vp, _vp, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong), _vp]
    lib.tt_bvh_load.argtypes = [_vp, _vp, ctypes.c_ulonglong, _vp, ctypes.c_int, _vp, ctypes.c_int, _vp]
    lib.tt_secondary_tree.argtypes = [_vp, _vp, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_int), _vp]
    lib.tt_mlp_update.argtypes = [_vp, ctypes.POINTER(TtMlp), _vp]
    lib.tt_mlp_train_step.argtypes = [_vp, ctypes.POINTER(TtMlp), ctypes.POINTER(TtMlpStep), _vp, _vp, ctypes.c_int,
                                      _vp, _vp]
    lib.tt_mlp_predict.argtypes = [_vp, ctypes.POINTER(TtMlp), _vp, ctypes.c_int, _vp, _vp]
    lib.tt_mlp_intervals.argtypes = [_vp, ctypes.POINTER(TtMlp), ctypes.POINTER(TtView), ctypes.c_int,
                                     ctypes.POINTER(_vp), ctypes.c_float, ctypes.c_float, ctypes.c_float, _vp]
    lib.tt_hit_cache_bytes.argtypes = [_vp, ctypes.c_longlong]
    lib.tt_hit_cache_bytes_pool.argtypes = [_vp, ctypes.c_longlong, ctypes.c_longlong]
    lib.tt_camera_rays.argtypes = [_vp, ctypes.POINTER(TtCamera), ctypes.c_int, _vp]
    lib.tt_hit_cache_usage.argtypes = [_vp, _vp, _vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]
    for name in EXPORTS:
        getattr(lib, name).restype = getattr(lib, name).restype if name == "tt_last_error" else ctypes.c_int
    lib.tt_hit_cache_bytes.restype = ctypes.c_size_t
    lib.tt_hit_cache_bytes_pool.restype = ctypes.c_size_t
    return lib


lib = _load()


class TracerError(RuntimeError):
    """Raised for a failed C-ABI call (RuntimeError, like the reference's
    exceptions through pybind11)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(handle, rc: int):
    if rc != TT_OK:
        msg = lib.tt_last_error(handle).decode(errors="replace") if handle else f"tritracer error {rc}"
        raise TracerError(rc, msg)
