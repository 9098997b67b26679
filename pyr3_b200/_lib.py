"""ctypes binding of libpyr3cuda.so (the C-ABI in include/pyr3.h).

The shared library is built in-tree by pyr3_b200/build.py.  There is no
CPU fallback: if the library is missing or cannot be loaded, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyr3cuda.so")

PYR3_OK = 0
PYR3_E_INVALID = -1
PYR3_E_CUDA = -2
PYR3_E_NVRTC = -3
PYR3_E_NOMEM = -4
PYR3_E_UNSUPPORTED = -5
OUT_RGBA8 = 0
OUT_RGBA32F = 1
OUT_RGBA16F = 2
OUT_PNG16 = 3
OUT_EXR_DISPLAY = 4
ITER_EXACT_WALKERS = 1
ITER_AGGREGATE = 2
ITER_KERNEL_BARRIER = 4
ITER_KERNEL_QUEUE = 8
ITER_KERNEL_WAVE = 16


class Pyr3Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"pyr3 error {code}: {msg}")
        self.code = code


class Opts(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("oversample", C.c_uint32),
                ("filter_radius", C.c_float), ("device", C.c_int32)]


class GenomeC(C.Structure):
    _fields_ = [("xforms", C.c_void_p), ("n_xforms", C.c_uint32), ("final_slot", C.c_int32),
                ("xaos", C.c_void_p), ("scale", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("rotate_deg", C.c_float), ("palette_mode", C.c_uint32),
                ("xform_blend", C.c_float)]


class IterateOpts(C.Structure):
    _fields_ = [("walkers", C.c_uint64), ("iters_per_walker", C.c_uint64), ("seed", C.c_uint32),
                ("walker_jitter", C.c_float), ("color_mode", C.c_uint32),
                ("flow_strength", C.c_float), ("flow_scale", C.c_float),
                ("trap_kind", C.c_uint32), ("trap_mode", C.c_uint32), ("trap_cx", C.c_float),
                ("trap_cy", C.c_float), ("trap_radius", C.c_float), ("trap_angle_deg", C.c_float),
                ("trap_falloff", C.c_float), ("trap_freq", C.c_float),
                ("trap_strength", C.c_float), ("phase_strength", C.c_float),
                ("phase_freq", C.c_float), ("flags", C.c_uint32)]


class PresentOpts(C.Structure):
    _fields_ = [("gamma", C.c_float), ("vibrancy", C.c_float), ("highpow", C.c_float),
                ("brightness", C.c_float), ("linrange", C.c_float), ("density_on", C.c_int32),
                ("de_max_rad", C.c_float), ("de_min_rad", C.c_float), ("de_curve", C.c_float),
                ("background", C.c_float * 3), ("transparent", C.c_int32), ("scale", C.c_double),
                ("curves_active", C.c_uint32), ("curves", C.c_void_p), ("hsl_active", C.c_int32),
                ("hsl_hue", C.c_float), ("hsl_sat", C.c_float), ("hsl_light", C.c_float)]


class BrightnessFit(C.Structure):
    """pyr3_brightness_fit: BrightnessFit (src/auto-exposure.ts:131-142)."""
    _fields_ = [("brightness", C.c_double), ("corrected", C.c_int32), ("iters", C.c_int32),
                ("final_mean", C.c_double), ("factor", C.c_double)]


# int rerender(double brightness, double *mean, void *ctx)
RERENDER_FN = C.CFUNCTYPE(C.c_int, C.c_double, C.POINTER(C.c_double), C.c_void_p)

# name -> (restype, argtypes)
_SIGS = {
    "pyr3_create": (C.c_int, [C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "pyr3_destroy": (C.c_int, [C.c_void_p]),
    "pyr3_resize": (C.c_int, [C.c_void_p, C.POINTER(Opts)]),
    "pyr3_last_error": (C.c_char_p, []),
    "pyr3_reset": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pyr3_iterate": (C.c_int, [C.c_void_p, C.POINTER(GenomeC), C.POINTER(IterateOpts)]),
    "pyr3_present": (C.c_int, [C.c_void_p, C.POINTER(PresentOpts), C.c_uint64, C.c_void_p, C.c_int32]),
    "pyr3_present_device": (C.c_int, [C.c_void_p, C.POINTER(PresentOpts), C.c_uint64, C.c_void_p,
                                      C.c_int32]),
    "pyr3_read_histogram": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pyr3_read_index_map": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pyr3_set_capture_index": (C.c_int, [C.c_void_p, C.c_int32]),
    "pyr3_sync": (C.c_int, [C.c_void_p]),
    "pyr3_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                            C.POINTER(C.c_void_p)]),
    "pyr3_counters": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "pyr3_last_iterate_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "pyr3_last_iterate_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "pyr3_dn_conv3x3": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_int64, C.c_int32,
                                  C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                  C.c_void_p]),
    "pyr3_dn_conv3x3_bf16": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_int64, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                       C.c_void_p]),
    "pyr3_dn_conv3x3_wgrad": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_int64, C.c_int32,
                                        C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_uint64, C.c_void_p]),
    "pyr3_dn_wgrad_scratch_floats": (C.c_uint64, [C.c_int32, C.c_int32]),
    "pyr3_splat_rate": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_float)]),
    "pyr3_dn_conv3x3_wgrad_bf16": (C.c_int, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_int64, C.c_int32,
                                             C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_uint64, C.c_void_p]),
    "pyr3_dn_flip_weights": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "pyr3_dn_relu_mask": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                    C.c_int32, C.c_void_p]),
    "pyr3_dn_add": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                              C.c_void_p]),
    "pyr3_dn_pool2": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                                C.c_int32, C.c_int32, C.c_int32, C.c_void_p]),
    "pyr3_dn_up2": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                              C.c_int32, C.c_int32, C.c_void_p]),
    "pyr3_dn_mse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pyr3_dn_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float,
                               C.c_float, C.c_float, C.c_int32, C.c_void_p]),
    "pyr3_mark": (C.c_int, [C.c_void_p, C.c_int32]),
    "pyr3_elapsed": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_float)]),
    "pyr3_flush_l2": (C.c_int, [C.c_void_p, C.c_uint64]),
    "pyr3_seed_walkers": (C.c_int, [C.c_uint32, C.c_uint64, C.c_uint32, C.c_void_p]),
    "pyr3_eval_variation": (C.c_int, [C.c_uint32, C.c_uint32, C.c_void_p, C.c_float, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pyr3_eval_dc_color": (C.c_int, [C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    "pyr3_pick_stream": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "pyr3_splat_points": (C.c_int, [C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float,
                                    C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_void_p,
                                    C.c_int32, C.c_void_p]),
    "pyr3_density_tonemap": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                       C.POINTER(PresentOpts), C.c_uint64, C.c_void_p, C.c_void_p]),
    "pyr3_density_tonemap_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                               C.c_float, C.POINTER(PresentOpts), C.c_uint64,
                                               C.c_void_p, C.c_int32, C.c_void_p]),
    "pyr3_prepare": (C.c_int, [C.c_void_p, C.POINTER(GenomeC)]),
    "pyr3_read_linear": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_void_p]),
    "pyr3_convert_display": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p]),
    "pyr3_fit_brightness": (C.c_int, [C.c_double, C.c_double, C.c_double, RERENDER_FN, C.c_void_p,
                                      C.POINTER(BrightnessFit)]),
    "pyr3_mean_luminance": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32,
                                      C.POINTER(C.c_double)]),
    "pyr3_auto_exposure": (C.c_int, [C.c_void_p, C.POINTER(PresentOpts), C.c_uint64, C.c_double,
                                     C.c_void_p, C.c_int32, C.POINTER(BrightnessFit)]),
    "pyr3_batch_create": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                    C.POINTER(C.c_void_p)]),
    "pyr3_batch_run": (C.c_int, [C.c_void_p]),
    "pyr3_batch_sync": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint64)]),
    "pyr3_batch_destroy": (C.c_int, [C.c_void_p]),
    "pyr3_jit_compile": (C.c_int, [C.POINTER(GenomeC), C.c_int32, C.POINTER(C.c_uint64)]),
    "pyr3_jit_source": (C.c_int, [C.POINTER(GenomeC), C.c_char_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "pyr3_jit_compile_variation": (C.c_int, [C.c_uint32, C.POINTER(C.c_uint64)]),
    "pyr3_pick_table": (C.c_int, [C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "pyr3_variation_info": (C.c_int, [C.c_uint32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                      C.POINTER(C.c_char_p)]),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise Pyr3Error(PYR3_E_CUDA, f"{LIB_PATH} is missing: run `python -m pyr3_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != PYR3_OK:
        raise Pyr3Error(rc, lib().pyr3_last_error().decode(errors="replace"))


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def exported_symbols() -> list:
    return sorted(_SIGS)
