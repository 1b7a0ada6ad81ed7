"""ctypes mirror of include/lambda_gpu.h and the loader for liblambda_b200.so.

The library is built in-tree by lambda_b200/build.py. Loading fails loudly when it
is missing: there is no Python or CPU fallback for any entry point.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblambda_b200.so")

CIE_BINS = 471
HERO_COUNT = 4
MLP_PARAMS = 8964

# lambda_status
STATUS_NAMES = {
    0: "LAMBDA_OK",
    1: "LAMBDA_ERR_INVALID_ARGUMENT",
    2: "LAMBDA_ERR_PARSE",
    3: "LAMBDA_ERR_IO",
    4: "LAMBDA_ERR_CUDA",
    5: "LAMBDA_ERR_OUT_OF_MEMORY",
    6: "LAMBDA_ERR_NO_SCENE",
    7: "LAMBDA_ERR_UNSUPPORTED",
    8: "LAMBDA_ERR_QUEUE_OVERFLOW",
    9: "LAMBDA_ERR_TIMEOUT",
    10: "LAMBDA_ERR_ABORTED",
    11: "LAMBDA_ERR_INTERNAL",
}

RENDER_THINFILM_EXACT = 0
RENDER_THINFILM_SURROGATE = 1
RENDER_OUTPUT_DEVICE = 2
RENDER_PROFILE_STAGES = 4
RENDER_THINFILM_FP64 = 8
NUM_STAGES = 14
PATH_KERNEL_PIXELS = 32768  # LAMBDA_PATH_KERNEL_PIXELS
# the surrogate's grazing region, where renders take the exact transfer matrix
SURROGATE_GRAZING_COS = 0.05  # LAMBDA_SURROGATE_GRAZING_COS
SURROGATE_LOW_SUB_INDEX = 1.05  # LAMBDA_SURROGATE_LOW_SUB_INDEX
SURROGATE_LOW_SUB_COS = 0.2  # LAMBDA_SURROGATE_LOW_SUB_COS
STAGE_NAMES = ("init", "wave_prologue", "raygen", "intersect", "shade_lambert", "shade_specular", "shade_film",
               "shadow", "finish", "film_encode", "film_mlp", "film_scatter", "path", "bounce")


class LambdaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Object(C.Structure):
    _fields_ = [("type", C.c_int32), ("material", C.c_int32), ("g", C.c_float * 27)]


class Instance(C.Structure):
    _fields_ = [("object", C.c_int32), ("count", C.c_int32), ("node", C.c_int32), ("material", C.c_int32),
                ("transform", C.c_float * 16), ("inverse_transform", C.c_float * 16)]


class BVHNode(C.Structure):
    _fields_ = [("min", C.c_float * 3), ("max", C.c_float * 3), ("index", C.c_int32), ("count", C.c_int32)]


class Material(C.Structure):
    _fields_ = [("type", C.c_int32), ("p", C.c_int32 * 3)]


class ScalarTexture(C.Structure):
    _fields_ = [("type", C.c_int32), ("p", C.c_float * 3)]


class SpectrumTexture(C.Structure):
    _fields_ = [("type", C.c_int32), ("value1", C.c_int32), ("value2", C.c_int32), ("scale", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("corner", C.c_float * 3), ("horizontal", C.c_float * 3),
                ("vertical", C.c_float * 3)]


class RenderSettings(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32), ("samples", C.c_int32),
                ("sqrt_samples", C.c_int32), ("lambda_min", C.c_float), ("lambda_max", C.c_float),
                ("camera", Camera)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("spectra", C.POINTER(C.c_float)), ("num_spectra", C.c_int32),
        ("complex_spectra", C.POINTER(C.c_double)), ("num_complex_spectra", C.c_int32),
        ("background_texture", C.c_int32),
        ("objects", C.POINTER(Object)), ("num_objects", C.c_int32),
        ("instances", C.POINTER(Instance)), ("num_instances", C.c_int32),
        ("nodes", C.POINTER(BVHNode)), ("num_nodes", C.c_int32),
        ("light_instances", C.POINTER(C.c_int32)), ("light_objects", C.POINTER(C.c_int32)),
        ("light_powers", C.POINTER(C.c_float)), ("num_lights", C.c_int32), ("total_light_power", C.c_float),
        ("materials", C.POINTER(Material)), ("num_materials", C.c_int32),
        ("material_properties", C.POINTER(C.c_int32)), ("num_material_properties", C.c_int32),
        ("scalar_textures", C.POINTER(ScalarTexture)), ("num_scalar_textures", C.c_int32),
        ("spectrum_textures", C.POINTER(SpectrumTexture)), ("num_spectrum_textures", C.c_int32),
    ]


class RenderDesc(C.Structure):
    _fields_ = [("settings", RenderSettings), ("seed", C.c_uint64), ("flags", C.c_uint32), ("reserved", C.c_int32)]


class Job(C.Structure):
    _fields_ = [("desc", RenderDesc), ("out_rgb", C.c_void_p)]


class Tuning(C.Structure):
    _fields_ = [("trace_block", C.c_int32), ("shade_block", C.c_int32), ("grid_scale", C.c_int32),
                ("max_pixels", C.c_int32), ("bvh_width", C.c_int32), ("path_kernel_pixels", C.c_int32),
                ("lane_fetch", C.c_int32), ("compressed_nodes", C.c_int32), ("fused_bounce", C.c_int32)]


class RenderStats(C.Structure):
    _fields_ = [("render_ms", C.c_double), ("paths", C.c_int64), ("segments", C.c_int64),
                ("shadow_rays", C.c_int64), ("thinfilm_hits", C.c_int64), ("thinfilm_fallback", C.c_int64),
                ("kernel_launches", C.c_int32), ("waves", C.c_int32), ("surrogate_ctas_per_sm", C.c_int32),
                ("reserved", C.c_int32)]


class StageTime(C.Structure):
    _fields_ = [("ms", C.c_double), ("launches", C.c_int64), ("items", C.c_int64)]


class FilmQuery(C.Structure):
    _fields_ = [("lambda_nm", C.c_float), ("cos_theta", C.c_float), ("thickness_nm", C.c_float),
                ("n_film", C.c_float), ("n_sub", C.c_float)]


class FilmRange(C.Structure):
    _fields_ = [("lambda_nm", C.c_float * 2), ("cos_theta", C.c_float * 2), ("thickness_nm", C.c_float * 2),
                ("n_film", C.c_float * 2), ("n_sub", C.c_float * 2)]


class TrainDesc(C.Structure):
    _fields_ = [("samples", C.c_int64), ("epochs", C.c_int32), ("batch", C.c_int32),
                ("learning_rate", C.c_float), ("seed", C.c_uint64), ("range", FilmRange)]


class Limits(C.Structure):
    """lambda_limits: device guard limits for tests that make a guard fire."""
    _fields_ = [("mma_polls", C.c_uint32), ("stack_entries", C.c_int32)]


DEFAULT_MMA_POLLS = 4194304  # LAMBDA_DEFAULT_MMA_POLLS


class TrainReport(C.Structure):
    _fields_ = [("train_ms", C.c_double), ("label_ms", C.c_double), ("final_loss", C.c_float),
                ("max_abs_error", C.c_float), ("mean_abs_error", C.c_float), ("audit_samples", C.c_int32)]


# name -> (restype, argtypes)
_P = C.c_void_p
_SIGNATURES = {
    "lambda_parse_lrd": (C.c_int, [C.c_char_p, C.POINTER(_P), C.c_char_p, C.c_size_t]),
    "lambda_parse_lrd_gpu": (C.c_int, [_P, C.c_char_p, C.c_int32, C.POINTER(_P), C.c_char_p, C.c_size_t]),
    "lambda_host_scene_get": (C.c_int, [_P, C.POINTER(SceneDesc), C.POINTER(RenderSettings)]),
    "lambda_host_scene_destroy": (None, [_P]),
    "lambda_write_ppm": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, _P, C.c_char_p, C.c_size_t]),
    "lambda_write_pfm": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, _P, C.c_int32, C.c_char_p, C.c_size_t]),
    "lambda_ctx_create": (C.c_int, [C.c_int32, C.POINTER(_P)]),
    "lambda_ctx_destroy": (None, [_P]),
    "lambda_last_error": (C.c_char_p, [_P]),
    "lambda_scene_upload": (C.c_int, [_P, C.POINTER(SceneDesc)]),
    "lambda_render": (C.c_int, [_P, C.POINTER(RenderDesc), _P, _P]),
    "lambda_render_batch": (C.c_int, [_P, C.POINTER(Job), C.c_int32, _P]),
    "lambda_autotune": (C.c_int, [_P, C.POINTER(RenderDesc), C.POINTER(Tuning)]),
    "lambda_autotune_batch": (C.c_int, [_P, C.POINTER(RenderDesc), C.c_int32, C.POINTER(Tuning)]),
    "lambda_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "lambda_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "lambda_set_limits": (C.c_int, [_P, C.POINTER(Limits)]),
    "lambda_get_limits": (C.c_int, [_P, C.POINTER(Limits)]),
    "lambda_get_render_stats": (C.c_int, [_P, C.POINTER(RenderStats)]),
    "lambda_get_stage_times": (C.c_int, [_P, C.POINTER(StageTime)]),
    "lambda_trace_closest": (C.c_int, [_P, _P, C.c_int32, _P, _P, _P]),
    "lambda_trace_shadow": (C.c_int, [_P, _P, _P, _P, C.c_int32, _P]),
    "lambda_thinfilm_exact": (C.c_int, [_P, _P, C.c_int32, _P]),
    "lambda_thinfilm_fp64": (C.c_int, [_P, _P, C.c_int32, _P]),
    "lambda_surrogate_train": (C.c_int, [_P, C.POINTER(TrainDesc), C.POINTER(TrainReport)]),
    "lambda_surrogate_set": (C.c_int, [_P, _P, C.POINTER(FilmRange)]),
    "lambda_surrogate_get": (C.c_int, [_P, _P, C.POINTER(FilmRange)]),
    "lambda_surrogate_eval": (C.c_int, [_P, _P, C.c_int32, _P]),
    "lambda_surrogate_grad": (C.c_int, [_P, _P, _P, _P, C.c_int32, _P, _P]),
    "lambda_surrogate_eval_static": (C.c_int, [_P, _P, C.c_int32, _P]),
}

EXPORTED_SYMBOLS = tuple(_SIGNATURES)

_lib = None


def load() -> C.CDLL:
    """Loads liblambda_b200.so from the package directory (built by build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run lambda_b200.build.build() (no fallback exists)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
