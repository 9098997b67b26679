"""Render-time auto-exposure (src/auto-exposure.ts) over the C-ABI.

The reference renders a cheap probe of the genome at the viewer's preview
geometry (1024 long edge, 16 spp, fixed seed), takes its mean luminance as
the target, then re-presents the high-quality histogram at refined
brightnesses until its mean luminance matches (bin/pyr3-render.ts:487-513).
Each of its passes reads the whole texture back to the host.  Here the
present, the luminance sum and the loop stay on the device: pyr3_auto_exposure
reads back 8 bytes per pass.

    target = measure_probe_luminance(genome)
    fit, image = auto_expose(renderer, genome, total_samples, target)
"""
from __future__ import annotations

import copy
import ctypes as C
import math
from dataclasses import dataclass

from . import _lib
from .genome import Genome
from .renderer import DEFAULT_FILTER_RADIUS, Renderer, compute_dispatch

# src/auto-exposure.ts:43-61 (PYR3_AE_* in include/pyr3.h)
AE_PROBE_LONG_EDGE = 1024
AE_PROBE_QUALITY = 16
AE_PROBE_SEED = 0x9E3779B9
AE_DEADBAND = 0.10
AE_MAX_ITERS = 4
AE_BRIGHTNESS_MIN = 1e-3
AE_BRIGHTNESS_MAX = 1e4


@dataclass
class BrightnessFit:
    """BrightnessFit (src/auto-exposure.ts:131-142)."""
    brightness: float
    corrected: bool
    iters: int
    final_mean: float
    factor: float


def _fit(c: _lib.BrightnessFit) -> BrightnessFit:
    return BrightnessFit(c.brightness, bool(c.corrected), c.iters, c.final_mean, c.factor)


def fit_brightness_to_target(base_brightness: float, target_mean: float, initial_mean: float,
                             rerender) -> BrightnessFit:
    """fitBrightnessToTarget (src/auto-exposure.ts:147-175), run by the
    library's fit logic; rerender(b) re-presents at brightness b and returns
    the measured mean luminance.  An exception in rerender ends the fit and
    is raised here."""
    err = []

    def cb(b, mean_p, _ctx):
        try:
            mean_p[0] = float(rerender(b))
            return 0
        except BaseException as e:  # noqa: BLE001 -- re-raised below
            err.append(e)
            return _lib.PYR3_E_INVALID

    fn = _lib.RERENDER_FN(cb)
    out = _lib.BrightnessFit()
    rc = _lib.lib().pyr3_fit_brightness(float(base_brightness), float(target_mean),
                                        float(initial_mean), fn, None, C.byref(out))
    if err:
        raise err[0]
    _lib.check(rc)
    return _fit(out)


def _after_torch(image) -> None:
    """The library works on the renderer's own stream: let the work torch
    has queued on the image's device (its producer, or a former owner of its
    memory) finish first."""
    import torch

    torch.cuda.current_stream(image.device).synchronize()


def _kind(image) -> int:
    import torch

    if image.dtype == torch.uint8:
        return _lib.OUT_RGBA8
    if image.dtype == torch.float32:
        return _lib.OUT_RGBA32F
    if image.dtype == torch.float16:
        return _lib.OUT_RGBA16F
    raise ValueError("image must be RGBA uint8, float16 or float32")


def mean_luminance(renderer: Renderer, image) -> float:
    """computeMeanLuminance / computeMeanLuminanceHalf (src/auto-exposure.ts:
    70-97) of an RGBA CUDA tensor (uint8: rgba8unorm; float16: the
    rgba16float texture; float32: read as that texture), computed on the
    device."""
    if not image.is_cuda or not image.is_contiguous() or image.numel() % 4:
        raise ValueError("image must be a contiguous RGBA CUDA tensor")
    _after_torch(image)
    out = C.c_double()
    _lib.check(_lib.lib().pyr3_mean_luminance(renderer.handle, C.c_void_p(image.data_ptr()),
                                              image.numel() // 4, _kind(image), C.byref(out)))
    return out.value


def apply_probe_preset(genome: Genome, long_edge: int = AE_PROBE_LONG_EDGE,
                       quality: int = AE_PROBE_QUALITY) -> Genome:
    """applyPreset(genome, customSpec(long_edge, quality)) (src/presets.ts:
    46-79, 128-136): force the long edge (short edge floored, aspect kept),
    scale and DE radii by the same factor, oversample 1, quality capped."""
    g = copy.deepcopy(genome)
    g.oversample = 1
    g.quality = min(genome.quality if genome.quality is not None else quality, quality)
    if genome.size is None:
        return g
    w, h = genome.size
    m = max(w, h)
    k = long_edge / m
    nw = long_edge if w == m else max(1, math.floor((long_edge * w) / h))
    nh = long_edge if h == m else max(1, math.floor((long_edge * h) / w))
    g.size = (nw, nh)
    g.scale = genome.scale * k
    if k != 1:  # scaleOutputPixelRadii (src/presets.ts:13-32)
        if genome.density is not None:
            g.density = dict(genome.density, maxRad=genome.density["maxRad"] * k,
                             minRad=genome.density["minRad"] * k)
        if genome.filter_radius is not None:
            g.filter_radius = genome.filter_radius * k
    return g


def measure_probe_luminance(genome: Genome, long_edge: int = AE_PROBE_LONG_EDGE,
                            quality: int = AE_PROBE_QUALITY, seed: int = AE_PROBE_SEED,
                            device: int = 0, renderer: Renderer | None = None) -> float:
    """measureProbeLuminance (src/auto-exposure.ts:99-129): render the
    genome at the preview geometry (oversample 1, the default spatial
    filter, fixed seed) into an rgba8 device image and return its mean
    luminance, the auto-exposure target.  The reference builds and destroys
    a renderer per probe; a caller that probes repeatedly can pass one to
    reuse (it is resized to the probe's geometry)."""
    import torch

    probe = apply_probe_preset(genome, long_edge, quality)
    w, h = probe.size if probe.size else (long_edge, long_edge)
    own = renderer is None
    if own:
        r = Renderer(w, h, 1, device=device)
    else:
        r = renderer
        if (r.width, r.height, r.oversample, r.filter_radius) != (w, h, 1, DEFAULT_FILTER_RADIUS):
            r.resize(w, h, 1, DEFAULT_FILTER_RADIUS)
    try:
        walkers, iters, samples = compute_dispatch(probe.quality, w, h)
        r.reset(probe)
        r.iterate(probe, seed, walkers, iters)
        img = torch.empty((h, w, 4), dtype=torch.uint8, device=torch.device("cuda", r.device))
        _after_torch(img)
        r.present_device(probe, samples, img.data_ptr())
        return mean_luminance(r, img)
    finally:
        if own:
            r.destroy()


def auto_expose(renderer: Renderer, genome: Genome, total_samples: int, target_mean: float,
                image=None, fmt: str = "rgba8", force_de_off: bool = False,
                transparent: bool = False):
    """The re-present loop of bin/pyr3-render.ts:487-513 on the device:
    present at the genome's brightness, measure, refine.  fmt "rgba8", "f16"
    (the rgba16float texture of the png16 / exr exports) or "f32".  Returns
    the fit and the CUDA image (H x W x 4) at fit.brightness."""
    import torch

    kind = {"rgba8": _lib.OUT_RGBA8, "f32": _lib.OUT_RGBA32F, "f16": _lib.OUT_RGBA16F}[fmt]
    if image is None:
        dtype = {_lib.OUT_RGBA8: torch.uint8, _lib.OUT_RGBA32F: torch.float32,
                 _lib.OUT_RGBA16F: torch.float16}[kind]
        image = torch.empty((renderer.height, renderer.width, 4), dtype=dtype,
                            device=torch.device("cuda", renderer.device))
    elif _kind(image) != kind or image.numel() != renderer.width * renderer.height * 4:
        raise ValueError("image does not match the renderer's size and format")
    _after_torch(image)
    p = renderer.present_opts(genome, force_de_off, transparent)
    out = _lib.BrightnessFit()
    _lib.check(_lib.lib().pyr3_auto_exposure(renderer.handle, C.byref(p), int(total_samples),
                                             float(target_mean), C.c_void_p(image.data_ptr()), kind,
                                             C.byref(out)))
    return _fit(out), image
