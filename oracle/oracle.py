"""ctypes bindings for the oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries:
* liboracle.so      (oracle/oracle.c): the C restatement of the reference's
  host algorithms and of the splat / density / visualize arithmetic;
* _ref/libpyr3_ref.so (the reference's own WGSL compiled for the CPU by
  oracle/wgsl2cpp.py): every variation, the chaos walker loop, density and
  visualize exactly as the reference's shaders state them;
* _ref/libpyr3_ref64.so: the same chaos shader evaluated in FP64.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GRAIN = 16384

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from oracle import build  # noqa: PLC0415

            build.build_oracle()
        L = C.CDLL(path)
        L.or_isaac_round.argtypes = [_u32p]
        L.or_irandinit.argtypes = [_u32p, C.c_int]
        L.or_isaac_irand.argtypes = [_u32p]
        L.or_isaac_irand.restype = C.c_uint32
        L.or_rand01.argtypes = [_u32p]
        L.or_rand01.restype = C.c_float
        L.or_rand_11.argtypes = [_u32p]
        L.or_rand_11.restype = C.c_float
        L.or_pack_isaac_states.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, _u32p]
        L.or_pack_xform_distrib.argtypes = [C.c_int, _f64p, C.c_void_p, _u32p]
        L.or_pack_xform_distrib.restype = C.c_int
        L.or_bake_lut.argtypes = [C.c_int, _f64p, _f64p, _f64p, _f64p, C.c_int, _f32p]
        L.or_derive_calibration.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int,
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.or_kernel_norm_lut.argtypes = [_f32p]
        L.or_spatial_kernel_gaussian.argtypes = [C.c_double, C.c_int, _f32p]
        L.or_spatial_kernel_gaussian.restype = C.c_int
        L.or_compute_dispatch.argtypes = [C.c_double, C.c_int, C.c_int, C.c_double] + \
            [C.POINTER(C.c_double)] * 3
        L.or_splat_points.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_float, C.c_float,
                                      C.c_float, C.c_float, C.c_int, _f32p, _u32p]
        L.or_pick_stream.argtypes = [C.c_int, _u32p, C.c_int, _i32p, _u32p, _u32p]
        L.or_density.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                 C.c_float, _f32p, _u32p, _f32p, C.c_int, C.c_int]
        L.or_visualize.argtypes = [C.c_void_p, _f32p, C.c_void_p, C.c_void_p, _f32p, C.c_int,
                                   C.c_int]
        L.or_histogram_to_linear.argtypes = [_u32p, C.c_int, C.c_int, C.c_int, C.c_double,
                                             C.c_double, _f32p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libpyr3_ref.so"))


def ref():
    """The reference's WGSL compiled for the CPU (oracle/_ref)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libpyr3_ref.so")
        if not os.path.exists(path):
            from oracle import build  # noqa: PLC0415

            build.build_reference()
        R = C.CDLL(path)
        R.ref_eval_variation.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float, _f32p,
                                         _f32p, _f32p, _u32p, _f32p]
        R.ref_eval_variation_grid.argtypes = [C.c_uint32, C.c_int, _f32p, C.c_float, _f32p,
                                              _f32p, _f32p, _u32p, _f32p]
        R.ref_dc_color.argtypes = [C.c_uint32, C.c_float, C.c_float, _f32p, _f32p, _f32p]
        R.ref_dc_color.restype = C.c_int
        R.ref_chaos_run.argtypes = [_u32p, _f32p, C.c_int, _f32p, _u32p, _u32p, C.c_uint32,
                                    C.c_uint32, _u32p, C.c_int]
        R.ref_chaos_run_capture.argtypes = [_u32p, _f32p, C.c_int, _f32p, _u32p, _u32p, C.c_uint32,
                                            C.c_uint32, _u32p, _u32p, C.c_int]
        R.ref_density.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float,
                                  C.c_float, C.c_float, _f32p, _u32p, _f32p, C.c_int]
        R.ref_visualize.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_float, C.c_float,
                                    C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_uint32,
                                    _f32p, C.c_uint32, _f32p, C.c_void_p, C.c_void_p, _f32p,
                                    C.c_int, C.c_uint32, C.c_void_p, C.c_uint32, C.c_float,
                                    C.c_float, C.c_float]
        _ref = R
    return _ref


_ref64 = None


def ref64():
    """The reference's chaos shader evaluated in FP64 (oracle/_ref/libpyr3_ref64.so)."""
    global _ref64
    if _ref64 is None:
        path = os.path.join(HERE, "_ref", "libpyr3_ref64.so")
        if not os.path.exists(path):
            from oracle import build  # noqa: PLC0415

            build.build_reference_f64()
        R = C.CDLL(path)
        R.ref64_eval_variation_grid.argtypes = [C.c_uint32, C.c_int, _f32p, C.c_float, _f32p, _f32p,
                                                _f32p, _u32p, _f64p]
        _ref64 = R
    return _ref64


# ----------------------------------------------------------------- helpers

def isaac_state(cnt, a, b, c, mem, rsl) -> np.ndarray:
    s = np.zeros(36, np.uint32)
    s[0], s[1], s[2], s[3] = cnt, a, b, c
    s[4:20] = mem
    s[20:36] = rsl
    return s


def pack_isaac_states(walkers: int, seed: int, base: int = 0) -> np.ndarray:
    out = np.zeros(walkers * 36, np.uint32)
    lib().or_pack_isaac_states(walkers, seed & 0xFFFFFFFF, base, out)
    return out


def pack_xform_distrib(weights, xaos=None) -> np.ndarray:
    n = len(weights)
    w = np.ascontiguousarray(weights, np.float64)
    rows = np.zeros((n + 1) * GRAIN, np.uint32)
    xp = None
    if xaos is not None:
        xa = np.ascontiguousarray(xaos, np.float64).reshape(n * n)
        xp = xa.ctypes.data
    rc = lib().or_pack_xform_distrib(n, w, xp, rows)
    if rc != 0:
        raise ValueError("xform weight must be non-negative finite")
    return rows


def bake_lut(stops, mode=0) -> np.ndarray:
    st = np.ascontiguousarray([s[0] for s in stops], np.float64)
    r = np.ascontiguousarray([s[1] for s in stops], np.float64)
    g = np.ascontiguousarray([s[2] for s in stops], np.float64)
    b = np.ascontiguousarray([s[3] for s in stops], np.float64)
    out = np.zeros(1024, np.float32)
    lib().or_bake_lut(len(stops), st, r, g, b, mode, out)
    return out


def derive_calibration(scale, samples, brightness, oversample=1):
    k1, k2 = C.c_double(), C.c_double()
    lib().or_derive_calibration(scale, samples, brightness, oversample, C.byref(k1), C.byref(k2))
    return k1.value, k2.value


def kernel_norm_lut() -> np.ndarray:
    out = np.zeros(257, np.float32)
    lib().or_kernel_norm_lut(out)
    return out


def spatial_kernel(radius=0.5, oversample=1) -> np.ndarray:
    out = np.zeros(17, np.float32)
    n = lib().or_spatial_kernel_gaussian(radius, oversample, out)
    if n < 0:
        raise ValueError("bad spatial filter args")
    return out[:n].copy()


def compute_dispatch(spp, width, height, walkers_override=0):
    w, i, s = C.c_double(), C.c_double(), C.c_double()
    lib().or_compute_dispatch(spp, width, height, walkers_override, C.byref(w), C.byref(i),
                              C.byref(s))
    return int(w.value), int(i.value), int(s.value)


def splat_points(pts, width, height, scale, cx, cy, rotation, palette_mode, palette, hist=None):
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1)
    if hist is None:
        hist = np.zeros(width * height * 4, np.uint32)
    lib().or_splat_points(len(pts) // 4, pts, width, height, scale, cx, cy, rotation,
                          palette_mode, np.ascontiguousarray(palette, np.float32), hist)
    return hist


def pick_stream(n, rows, prev, draws) -> np.ndarray:
    prev = np.ascontiguousarray(prev, np.int32)
    draws = np.ascontiguousarray(draws, np.uint32)
    out = np.zeros(len(draws), np.uint32)
    lib().or_pick_stream(n, rows, len(draws), prev, draws, out)
    return out


def density(hist, width, height, max_rad, min_rad, curve, k1, k2):
    out = np.zeros(width * height * 4, np.float32)
    lib().or_density(width, height, max_rad, min_rad, curve, k1, k2, kernel_norm_lut(),
                     np.ascontiguousarray(hist, np.uint32), out, 0, height)
    return out


class _Viz(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("oversample", C.c_int),
                ("fwidth", C.c_int), ("k1", C.c_float), ("k2", C.c_float),
                ("gamma", C.c_float), ("vibrancy", C.c_float), ("highpow", C.c_float),
                ("linrange", C.c_float), ("bg", C.c_float * 3), ("transparent", C.c_int),
                ("curves_active", C.c_uint), ("curves", C.c_void_p), ("hsl_active", C.c_int),
                ("hsl_hue", C.c_float), ("hsl_sat", C.c_float), ("hsl_light", C.c_float)]


def visualize(width, height, oversample, kernel, k1, k2, gamma, vibrancy, highpow, linrange,
              bg=(0, 0, 0), transparent=False, src_u32=None, src_f32=None, curves_active=0,
              curves=None, hsl=None):
    """hsl = (hue degrees, sat multiplier, light addend) or None."""
    cv = np.ascontiguousarray(curves, np.float32) if curves is not None else None
    v = _Viz(width, height, oversample, len(kernel), k1, k2, gamma, vibrancy, highpow, linrange,
             (C.c_float * 3)(*bg), int(transparent), int(curves_active),
             cv.ctypes.data if cv is not None else None, 1 if hsl else 0,
             *(hsl if hsl else (0.0, 1.0, 0.0)))
    out = np.zeros(width * height * 4, np.float32)
    su = np.ascontiguousarray(src_u32, np.uint32) if src_u32 is not None else None
    sf = np.ascontiguousarray(src_f32, np.float32) if src_f32 is not None else None
    lib().or_visualize(C.byref(v), np.ascontiguousarray(kernel, np.float32),
                       su.ctypes.data if su is not None else None,
                       sf.ctypes.data if sf is not None else None, out, 0, height)
    return out


def histogram_to_linear(hist, width, height, oversample, k1, k2):
    out = np.zeros(width * height * 4, np.float32)
    lib().or_histogram_to_linear(np.ascontiguousarray(hist, np.uint32), width, height,
                                 oversample, k1, k2, out)
    return out


# ------------------------------------------------------- reference shaders

def ref_eval_grid(idx, pts, w, params10, a0, a1, isaac):
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1)
    out = np.zeros_like(pts)
    ref().ref_eval_variation_grid(idx, len(pts) // 2, pts, w,
                                  np.ascontiguousarray(params10, np.float32),
                                  np.ascontiguousarray(a0, np.float32),
                                  np.ascontiguousarray(a1, np.float32), isaac, out)
    return out.reshape(-1, 2)


def ref64_eval_grid(idx, pts, w, params10, a0, a1, isaac):
    """apply_variation of the reference's shader evaluated in FP64 (f32
    inputs, double outputs), isaac advanced in place."""
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1)
    out = np.zeros(len(pts), np.float64)
    ref64().ref64_eval_variation_grid(idx, len(pts) // 2, pts, w,
                                      np.ascontiguousarray(params10, np.float32),
                                      np.ascontiguousarray(a0, np.float32),
                                      np.ascontiguousarray(a1, np.float32), isaac, out)
    return out.reshape(-1, 2)


def ref_dc_color(idx, px, py, v4, ve4):
    rgb = np.zeros(3, np.float32)
    hit = ref().ref_dc_color(idx, px, py, np.ascontiguousarray(v4, np.float32),
                             np.ascontiguousarray(ve4, np.float32), rgb)
    return bool(hit), rgb


def ref_chaos_run(uniforms31, xforms, n_std, palette, distrib, isaac, w0, w1, hist, threads):
    ref().ref_chaos_run(np.ascontiguousarray(uniforms31, np.uint32),
                        np.ascontiguousarray(xforms, np.float32), n_std,
                        np.ascontiguousarray(palette, np.float32),
                        np.ascontiguousarray(distrib, np.uint32), isaac, w0, w1, hist, threads)


def ref_chaos_run_capture(uniforms31, xforms, n_std, palette, distrib, isaac, w0, w1, hist, idx_sum,
                          threads):
    """ref_chaos_run with the capture-index pass on (uniforms31[14] = 1)."""
    ref().ref_chaos_run_capture(np.ascontiguousarray(uniforms31, np.uint32),
                                np.ascontiguousarray(xforms, np.float32), n_std,
                                np.ascontiguousarray(palette, np.float32),
                                np.ascontiguousarray(distrib, np.uint32), isaac, w0, w1, hist, idx_sum,
                                threads)


def ref_density(hist, width, height, max_rad, min_rad, curve, k1, k2, threads=8):
    out = np.zeros(width * height * 4, np.float32)
    ref().ref_density(width, height, max_rad, min_rad, curve, k1, k2, kernel_norm_lut(),
                      np.ascontiguousarray(hist, np.uint32), out, threads)
    return out


def ref_visualize(width, height, oversample, kernel, k1, k2, gamma, vibrancy, highpow, linrange,
                  bg=(0, 0, 0), transparent=False, src_u32=None, src_f32=None, threads=8,
                  curves_active=0, curves=None, hsl=None):
    out = np.zeros(width * height * 4, np.float32)
    su = np.ascontiguousarray(src_u32, np.uint32) if src_u32 is not None else None
    sf = np.ascontiguousarray(src_f32, np.float32) if src_f32 is not None else None
    cv = np.ascontiguousarray(curves, np.float32) if curves is not None else None
    h = hsl if hsl else (0.0, 1.0, 0.0)
    ref().ref_visualize(width, height, k1, k2, gamma, vibrancy, highpow, linrange, oversample,
                        len(kernel), np.ascontiguousarray(bg, np.float32), int(transparent),
                        np.ascontiguousarray(kernel, np.float32),
                        su.ctypes.data if su is not None else None,
                        sf.ctypes.data if sf is not None else None, out, threads,
                        int(curves_active), cv.ctypes.data if cv is not None else None,
                        1 if hsl else 0, h[0], h[1], h[2])
    return out
