"""ctypes binding of libwgpt.so (include/wgpt.h).

The library is the product: there is no CPU fallback.  If it is missing or cannot be loaded the
import raises, naming the build step (webgpuraytracer_b200.build.build()).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libwgpt.so"

WGPT_OK = 0
STATUS_NAMES = {
    0: "WGPT_OK", 1: "WGPT_E_INVALID", 2: "WGPT_E_LAYOUT", 3: "WGPT_E_CUDA", 4: "WGPT_E_NOMEM",
    5: "WGPT_E_STATE", 6: "WGPT_E_UNSUPPORTED", 7: "WGPT_E_REBUILD", 8: "WGPT_E_DEVICE",
    9: "WGPT_E_TOO_LARGE", 10: "WGPT_E_TIMEOUT",
}
NOALLOC_MAX_PIXELS = 131072

MODE_WAVEFRONT = 0
MODE_MEGAKERNEL = 1
ENV_CDF = 0
ENV_ALIAS = 1

# feature flags (pipeline override constants 1..11, shader.wgsl:1-12)
HAS_SPHERES = 1 << 0
HAS_CUBES = 1 << 1
HAS_PLANES = 1 << 2
HAS_CYLINDERS = 1 << 3
HAS_TORI = 1 << 4
HAS_MESHES = 1 << 5
HAS_LIST_MESHES = 1 << 6
HAS_HEIGHTMAPS = 1 << 7
HAS_LIGHTS = 1 << 8
HAS_SKYBOX = 1 << 9
MIS_SKYBOX = 1 << 10


class Buffer(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("bytes", C.c_size_t)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("materials", Buffer), ("objects", Buffer), ("tlas", Buffer), ("meshes", Buffer), ("bvh", Buffer),
        ("triangles", Buffer), ("planes", Buffer), ("lights", Buffer), ("sky_cdf", Buffer),
        ("sky_rgba16f", C.c_void_p), ("sky_width", C.c_uint32), ("sky_height", C.c_uint32),
        ("bounce_limit", C.c_int32), ("feature_flags", C.c_uint32),
        ("textures_rgba8", C.c_void_p), ("tex_width", C.c_uint32), ("tex_height", C.c_uint32),
        ("tex_layers", C.c_uint32), ("sky_alias", C.c_void_p),
    ]


class WavefrontTuning(C.Structure):
    _fields_ = [("trav_shape", C.c_uint32), ("shade_block", C.c_uint32), ("refill_closest", C.c_uint32),
                ("refill_shadow", C.c_uint32), ("shadow_wide", C.c_uint32)]


class WgptError(RuntimeError):
    def __init__(self, code: int, what: str, msg: str = ""):
        self.code = code
        super().__init__(f"{what}: {STATUS_NAMES.get(code, code)}" + (f" ({msg})" if msg else ""))


_P = C.c_void_p
_U32 = C.c_uint32
_I32 = C.c_int32
_F = C.c_float

EXPORTS = {
    "wgpt_abi_version": ([], C.c_int),
    "wgpt_create": ([C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "wgpt_destroy": ([_P], C.c_int),
    "wgpt_last_error": ([_P], C.c_char_p),
    "wgpt_validate_scene": ([C.POINTER(SceneDesc), C.c_char_p, C.c_size_t], C.c_int),
    "wgpt_upload_scene": ([_P, C.POINTER(SceneDesc)], C.c_int),
    "wgpt_update_scene": ([_P, C.POINTER(SceneDesc)], C.c_int),
    "wgpt_update_objects": ([_P, C.POINTER(SceneDesc)], C.c_int),
    "wgpt_resize": ([_P, _U32, _U32, C.c_int], C.c_int),
    "wgpt_set_params": ([_P, _P], C.c_int),
    "wgpt_render": ([_P, _U32, _U32, _U32, _U32, _U32, _U32], C.c_int),
    "wgpt_render_gbuffer": ([_P, _U32, _U32, _U32, _U32], C.c_int),
    "wgpt_denoise": ([_P, _P, _P, _U32], C.c_int),
    "wgpt_resample": ([_P, _U32, _U32, _F, _F], C.c_int),
    "wgpt_synchronize": ([_P], C.c_int),
    "wgpt_synchronize_timeout": ([_P, C.c_uint32], C.c_int),
    "wgpt_selftest_wait": ([C.c_int, C.c_uint32, _P, _P], C.c_int),
    "wgpt_read_accum": ([_P, _P], C.c_int),
    "wgpt_write_accum": ([_P, _P], C.c_int),
    "wgpt_read_output": ([_P, _P], C.c_int),
    "wgpt_read_gbuffer": ([_P, _P], C.c_int),
    "wgpt_write_gbuffer": ([_P, _P], C.c_int),
    "wgpt_read_denoised": ([_P, _P, _P], C.c_int),
    "wgpt_read_canvas": ([_P, _P, _U32, _U32], C.c_int),
    "wgpt_trace_rays": ([_P, _P, _U32, _P, _P, _P, _P, _P], C.c_int),
    "wgpt_set_render_mode": ([_P, C.c_int], C.c_int),
    "wgpt_set_env_sampling": ([_P, C.c_int], C.c_int),
    "wgpt_probe_l2_read": ([C.c_int, C.c_uint64, _U32, C.POINTER(C.c_double)], C.c_int),
    "wgpt_sample_env": ([_P, _P, _U32, _P, _P], C.c_int),
    "wgpt_set_denoise_mode": ([_P, C.c_int], C.c_int),
    "wgpt_kpcn_set_conv_mode": ([_P, C.c_int], C.c_int),
    "wgpt_set_wavefront_tuning": ([_P, _P], C.c_int),
    "wgpt_get_wavefront_tuning": ([_P, _P], C.c_int),
    "wgpt_rng_stream": ([C.c_int, _U32, _U32, _U32, _U32, _P], C.c_int),
    "wgpt_set_wavefront_config": ([_P, C.c_uint32, C.c_uint64], C.c_int),
    "wgpt_set_views": ([_P, C.c_uint32, _P, _P], C.c_int),
    "wgpt_set_accum_f64": ([_P, C.c_int], C.c_int),
    "wgpt_read_accum_f64": ([_P, _P], C.c_int),
    "wgpt_write_accum_f64": ([_P, _P], C.c_int),
    "wgpt_gemm_bf16": ([C.c_int, _P, _P, _P, C.c_int, C.c_int, C.c_int], C.c_int),
    "wgpt_kpcn_create": ([C.c_int, C.c_uint64, C.POINTER(_P)], C.c_int),
    "wgpt_kpcn_destroy": ([_P], C.c_int),
    "wgpt_kpcn_last_error": ([_P], C.c_char_p),
    "wgpt_kpcn_num_params": ([_P, C.POINTER(C.c_uint64)], C.c_int),
    "wgpt_kpcn_get_params": ([_P, _P], C.c_int),
    "wgpt_kpcn_set_params": ([_P, _P], C.c_int),
    "wgpt_kpcn_add_example": ([_P, _P, _P, _P, C.c_uint32, C.c_uint32], C.c_int),
    "wgpt_kpcn_num_examples": ([_P, C.POINTER(C.c_uint32)], C.c_int),
    "wgpt_kpcn_train": ([_P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_uint64, _P], C.c_int),
    "wgpt_kpcn_loss_and_grads": ([_P, _P, _P, _P, C.c_uint32, C.c_uint32, _P, _P, _P], C.c_int),
    "wgpt_kpcn_grads": ([_P, C.c_uint32, C.c_uint32, C.c_uint64, _P, _P], C.c_int),
    "wgpt_kpcn_apply": ([_P, _P, C.c_float, C.c_float], C.c_int),
    "wgpt_kpcn_denoise": ([_P, _P, C.c_float, _P], C.c_int),
    "wgpt_render_views": ([_P, _P, _P, _P, _P], C.c_int),
    "wgpt_read_view": ([_P, C.c_uint32, _P, _P], C.c_int),
    "wgpt_render_views_gbuffer": ([_P, _P], C.c_int),
    "wgpt_kpcn_denoise_view": ([_P, _P, C.c_uint32, C.c_float, _P], C.c_int),
    "wgpt_get_wavefront_config": ([_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)], C.c_int),
    "wgpt_denoise_noalloc": ([_P, _P, _P, _P, _U32, _P, _P, _P], C.c_int),
    "wgpt_set_counting": ([_P, C.c_int], C.c_int),
    "wgpt_read_counters": ([_P, _P], C.c_int),
    "wgpt_read_stage_counters": ([_P, _P], C.c_int),
    "wgpt_set_stage_timing": ([_P, C.c_int], C.c_int),
    "wgpt_read_stage_times": ([_P, _P, _P], C.c_int),
    "wgpt_stream": ([_P], C.c_void_p),
    "wgpt_build_blas": ([_P, _U32, _P, C.POINTER(_U32), _P], C.c_int),
    "wgpt_build_tlas": ([_P, _U32, _P, C.POINTER(_U32)], C.c_int),
    "wgpt_build_env_cdf": ([_P, _U32, _U32, C.c_double, _P, C.POINTER(C.c_double)], C.c_int),
    "wgpt_build_env_alias": ([_P, _U32, _U32, C.c_double, _P, _P], C.c_int),
    "wgpt_decode_rgbe": ([_P, C.c_size_t, C.c_double, _P, C.POINTER(_U32), C.POINTER(_U32)], C.c_int),
    "wgpt_parse_obj": ([_P, C.c_size_t, _P, C.c_uint32, C.POINTER(C.c_uint32), _P, C.c_uint32,
                        C.POINTER(C.c_uint32)], C.c_int),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Loads libwgpt.so once and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with webgpuraytracer_b200.build.build()")
    handle = C.CDLL(str(LIB_PATH))
    for name, (argtypes, restype) in EXPORTS.items():
        fn = getattr(handle, name)
        fn.argtypes = argtypes
        fn.restype = restype
    _lib = handle
    return handle


def ptr(a) -> int | None:
    """Address of a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the library must be C-contiguous"
    return a.ctypes.data


def check(rc: int, what: str, ctx=None) -> None:
    if rc != WGPT_OK:
        msg = ""
        if ctx is not None:
            raw = lib().wgpt_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise WgptError(rc, what, msg)
