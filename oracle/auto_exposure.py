"""CPU oracle of render-time auto-exposure -- TEST INFRASTRUCTURE ONLY (tests/
use it as the checker; the product never imports it).

A restatement of the reference's src/auto-exposure.ts in Python/numpy:
the mean-luminance measures (:70-97), the brightness fit (:147-175) and the
preview-probe geometry of applyPreset(customSpec(...)) (src/presets.ts:
13-32, 46-79, 128-136).  Pinned to the reference's own unit tests
(src/auto-exposure.test.ts), whose cases tests/test_auto_exposure.py runs
against this module and against the library.

The reference sums luminance left to right in float64; np.cumsum adds in the
same order, so its last element is the reference's sum bit for bit.
"""
from __future__ import annotations

import math

import numpy as np

# src/auto-exposure.ts:43-61
AE_PROBE_LONG_EDGE = 1024
AE_PROBE_QUALITY = 16
AE_PROBE_SEED = 0x9E3779B9
AE_DEADBAND = 0.10
AE_MAX_ITERS = 4
AE_BRIGHTNESS_MIN = 1e-3
AE_BRIGHTNESS_MAX = 1e4


def clamp(x: float, lo: float, hi: float) -> float:
    """src/auto-exposure.ts:63-70: non-finite -> lo."""
    return min(hi, max(lo, x)) if math.isfinite(x) else lo


def mean_luminance(pixels: np.ndarray) -> float:
    """computeMeanLuminance (src/auto-exposure.ts:72-79): mean of
    (R+G+B)/3 over rgba8 pixels, in [0, 255]; empty -> 0."""
    px = np.asarray(pixels, np.uint8).reshape(-1, 4)
    if len(px) == 0:
        return 0.0
    per = (px[:, 0].astype(np.float64) + px[:, 1] + px[:, 2]) / 3.0
    return float(np.cumsum(per)[-1] / len(px))


def mean_luminance_half(rgba_f16: np.ndarray) -> float:
    """computeMeanLuminanceHalf (src/auto-exposure.ts:84-97) of an
    rgba16float buffer: each channel clamped to [0, 1] (non-finite -> 0),
    (R+G+B)/3 * 255, averaged."""
    px = np.asarray(rgba_f16, np.float16).reshape(-1, 4).astype(np.float64)
    if len(px) == 0:
        return 0.0
    c = np.where(np.isfinite(px[:, :3]), np.clip(px[:, :3], 0.0, 1.0), 0.0)
    per = ((c[:, 0] + c[:, 1] + c[:, 2]) / 3.0) * 255.0
    return float(np.cumsum(per)[-1] / len(px))


def mean_luminance_rgba32f(rgba_f32: np.ndarray) -> float:
    """The rgba32f image as the reference would read it back from an
    rgba16float texture: rounded to binary16 (nearest even), then
    mean_luminance_half."""
    with np.errstate(over="ignore"):
        return mean_luminance_half(np.asarray(rgba_f32, np.float32).astype(np.float16))


def fit_brightness_to_target(base: float, target: float, initial: float, rerender):
    """fitBrightnessToTarget (src/auto-exposure.ts:147-175); rerender(b)
    returns the mean luminance at brightness b.  Returns (brightness,
    corrected, iters, final_mean, factor) and the brightnesses presented."""
    finite = math.isfinite(target) and math.isfinite(initial)
    factor0 = target / initial if finite and initial > 0 else 1.0
    if not finite or target <= 0 or initial <= 0 or abs(factor0 - 1) <= AE_DEADBAND:
        return (base, False, 0, initial, factor0), []
    b, mean, iters, seq = base, initial, 0, []
    for _ in range(AE_MAX_ITERS):
        factor = target / mean
        if abs(factor - 1) <= AE_DEADBAND:
            break
        b = clamp(b * factor, AE_BRIGHTNESS_MIN, AE_BRIGHTNESS_MAX)
        seq.append(b)
        mean = rerender(b)
        iters += 1
        if mean <= 0:
            break
    return (b, iters > 0, iters, mean, factor0), seq


def probe_geometry(size, scale: float, density, quality, long_edge: int = AE_PROBE_LONG_EDGE,
                   spp: int = AE_PROBE_QUALITY):
    """applyPreset(genome, customSpec(long_edge, spp)) (src/presets.ts:46-79,
    128-136) restricted to what the probe uses: returns (width, height,
    scale, density radii (max, min) or None, quality).  size is (w, h) or
    None; density is (max_rad, min_rad) or None."""
    capped = min(quality if quality is not None else spp, spp)
    if size is None:
        return long_edge, long_edge, scale, density, capped
    w, h = size
    m = max(w, h)
    k = long_edge / m
    nw = long_edge if w == m else max(1, math.floor((long_edge * w) / h))
    nh = long_edge if h == m else max(1, math.floor((long_edge * h) / w))
    if density is not None and k != 1:
        density = (density[0] * k, density[1] * k)
    return nw, nh, scale * k, density, capped
