"""CPU oracle of the display export transforms -- TEST INFRASTRUCTURE ONLY
(tests/ use it as the checker; the product never imports it).

Restates, in numpy, the reference's host-side transforms of its rgba16float
display readback: halfToFloat (src/half-float.ts:4-18), srgbToLinear
(src/srgb.ts:13-16), displayHalfToLinearExr (src/gpu-readback.ts:83-104)
and displayHalfToPng16 (src/gpu-readback.ts:106-115).  Pinned to the
reference's own cases (src/half-float.test.ts, src/srgb.test.ts,
src/gpu-readback.test.ts) in tests/test_display_formats.py.

JS arithmetic is IEEE double: srgbToLinear runs in float64 and the EXR
buffer (a Float32Array) rounds its result to float32 on store; png16's
Math.round(x) is floor(x + 0.5).
"""
from __future__ import annotations

import numpy as np


def half_to_float(bits) -> np.ndarray:
    """halfToFloat (src/half-float.ts:4-18) of binary16 bit patterns, as
    float64."""
    h = np.asarray(bits, np.uint32)
    sign = (h & 0x8000) >> 15
    exp = ((h & 0x7C00) >> 10).astype(np.int64)
    frac = (h & 0x03FF).astype(np.float64)
    with np.errstate(over="ignore", invalid="ignore"):
        val = np.where(exp == 0, frac * 2.0 ** -24,
                       np.where(exp == 0x1F, np.where(frac == 0, np.inf, np.nan),
                                (1 + frac / 1024) * np.power(2.0, (exp - 15).astype(np.float64))))
    return np.where(sign == 1, -val, val)


def to_half_bits(f32) -> np.ndarray:
    """The rgba16float texture of a fragment value: float32 -> binary16,
    round to nearest even (numpy's conversion), as bit patterns."""
    with np.errstate(over="ignore"):
        return np.asarray(f32, np.float32).astype(np.float16).view(np.uint16)


def srgb_to_linear(c) -> np.ndarray:
    """srgbToLinear (src/srgb.ts:13-16) in float64."""
    c = np.asarray(c, np.float64)
    with np.errstate(invalid="ignore"):
        return np.where(c <= 0.04045, c / 12.92, np.power((c + 0.055) / 1.055, 2.4))


def _cl(f: np.ndarray) -> np.ndarray:
    """The clamp of displayHalfToLinearExr: non-finite -> 0, else [0, 1];
    JS Math.max(0, -0) is +0, hence the + 0.0."""
    return np.where(np.isfinite(f), np.clip(f, 0.0, 1.0) + 0.0, 0.0)


def display_half_to_linear_exr(bits) -> np.ndarray:
    """displayHalfToLinearExr (src/gpu-readback.ts:83-104): n x 4 binary16
    bit patterns -> n x 4 float32 (sRGB-to-linear RGB, alpha clamped)."""
    f = half_to_float(np.asarray(bits).reshape(-1, 4))
    out = np.empty(f.shape, np.float32)
    out[:, :3] = srgb_to_linear(_cl(f[:, :3]))
    out[:, 3] = _cl(f[:, 3])
    return out


def display_half_to_png16(bits) -> np.ndarray:
    """displayHalfToPng16 (src/gpu-readback.ts:106-115): binary16 bit
    patterns -> uint16 samples round(clamp(f, 0, 1) * 65535); NaN -> 0 (the
    Uint16Array store of NaN)."""
    f = half_to_float(np.asarray(bits).reshape(-1, 4))
    with np.errstate(invalid="ignore"):
        x = np.floor(np.maximum(0.0, np.minimum(1.0, f)) * 65535.0 + 0.5)
    return np.where(np.isnan(f), 0, x).astype(np.uint16)
