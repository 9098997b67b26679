"""Host mirror of the reference's Renderer API (src/renderer.ts:163-318) over
the C-ABI: the same calls, argument meanings and error behaviour, with the
output view replaced by a host array (headless: no textures / swapchains).

    r = create_renderer(width=640, height=480, oversample=1)
    r.reset(genome)
    w, it, samples = compute_dispatch(spp, r.width, r.height)
    r.iterate(genome, seed=0, walkers=w, iters_per_walker=it)
    rgba8 = r.present(genome, total_samples=samples)
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .genome import (DEFAULT_TONEMAP, Genome, bake_curves, bake_lut, curves_active_mask,
                     expand_for_gpu, final_slot, pack_xforms, xaos_matrix)

# src/renderer.ts:23-47
DEFAULT_FILTER_RADIUS = 0.5
TARGET_WALKERS = 1024
MIN_ITERS_PER_WALKER = 4096
MAX_ITERS_PER_WALKER = 1048576
FUSE = 200
DEFAULT_SPP = 16
MAX_WALKERS = 65535 * 64
DEFAULT_WALKER_JITTER = 1e-7  # src/chaos.ts:96
DEFAULT_FLOW_SCALE = 2.0  # src/chaos.ts:139


# present() formats: name -> (PYR3_OUT_* kind, host dtype)
FORMATS = {"rgba8": (_lib.OUT_RGBA8, np.uint8), "f32": (_lib.OUT_RGBA32F, np.float32),
           "f16": (_lib.OUT_RGBA16F, np.float16), "png16": (_lib.OUT_PNG16, np.uint16),
           "exr": (_lib.OUT_EXR_DISPLAY, np.float32)}


def _js_round(x: float) -> int:
    return int(math.floor(x + 0.5))


def compute_dispatch(target_spp: float, width: int, height: int, walkers_override=None):
    """computeDispatch (src/renderer.ts:57-78) -> (walkers, iters, samples)."""
    target = _js_round(target_spp * width * height)
    walkers = walkers_override if walkers_override is not None else TARGET_WALKERS
    iters = math.ceil(target / walkers)
    if walkers_override is None:
        if iters < MIN_ITERS_PER_WALKER:
            iters = MIN_ITERS_PER_WALKER
            walkers = max(1, math.ceil(target / iters))
        elif iters > MAX_ITERS_PER_WALKER:
            iters = MAX_ITERS_PER_WALKER
            walkers = min(MAX_WALKERS, math.ceil(target / iters))
    else:
        iters = max(1, iters)
    return int(walkers), int(iters), int(walkers * iters)


class GpuGenome:
    """A genome packed for the C-ABI (keeps the numpy buffers alive)."""

    def __init__(self, genome: Genome):
        g = expand_for_gpu(genome)
        self.genome = g
        self.xforms = np.ascontiguousarray(pack_xforms(g), np.float32)
        xa = xaos_matrix(g)
        self.xaos = None if xa is None else np.ascontiguousarray(xa, np.float32)
        self.c = _lib.GenomeC(
            _lib.ptr(self.xforms), len(g.xforms), final_slot(g),
            _lib.ptr(self.xaos) if self.xaos is not None else None,
            g.scale, g.cx, g.cy, g.rotate or 0.0, 1 if g.palette_mode == "linear" else 0,
            min(1.0, max(0.0, g.xform_blend or 0.0)))


class Renderer:
    def __init__(self, width: int, height: int, oversample: int = 1, filter_radius=None,
                 device: int = 0):
        self._h = C.c_void_p()
        self._opts = _lib.Opts(width, height, max(1, int(oversample)),
                               filter_radius or DEFAULT_FILTER_RADIUS, device)
        _lib.check(_lib.lib().pyr3_create(C.byref(self._opts), C.byref(self._h)))
        self._capture = False
        self.launches = 0  # chaos-kernel launches issued by iterate() so far

    # ---- properties (src/renderer.ts:283-288)
    @property
    def width(self) -> int:
        return self._opts.width

    @property
    def height(self) -> int:
        return self._opts.height

    @property
    def oversample(self) -> int:
        return self._opts.oversample

    @property
    def filter_radius(self) -> float:
        return self._opts.filter_radius

    @property
    def super_w(self) -> int:
        return self.width * self.oversample

    @property
    def super_h(self) -> int:
        return self.height * self.oversample

    @property
    def handle(self):
        return self._h

    @property
    def device(self) -> int:
        """CUDA device ordinal the renderer lives on."""
        return self._opts.device

    # ---- API
    def reset(self, genome: Genome) -> None:
        """Upload the palette and zero the histogram (src/renderer.ts:221)."""
        lut = bake_lut(genome.palette, genome.palette_hue, genome.palette_interp)
        _lib.check(_lib.lib().pyr3_reset(self._h, _lib.ptr(lut)))

    def iterate(self, genome, seed: int, walkers: int, iters_per_walker: int,
                walker_jitter: float = DEFAULT_WALKER_JITTER, color_mode: str = "palette",
                flow_strength: float = 1.0, flow_scale: float = DEFAULT_FLOW_SCALE, trap=None,
                phase_strength: float = 1.0, phase_freq: float = 1.0, exact_walkers: bool = False,
                aggregate: bool = False, kernel: str = "auto") -> None:
        """Accumulate walkers x iters samples (src/renderer.ts:227).
        kernel: "auto" (the autotuner's choice), "barrier", "queue" or "wave"."""
        gg = genome if isinstance(genome, GpuGenome) else GpuGenome(genome)
        trap = trap or {}
        modes = {"palette": 0, "flow": 1, "trap-distance": 2, "phase": 3}
        o = _lib.IterateOpts(
            walkers, iters_per_walker, seed & 0xFFFFFFFF, walker_jitter, modes[color_mode],
            flow_strength, flow_scale,
            {"point": 0, "circle": 1, "line": 2}[trap.get("kind", "point")],
            1 if trap.get("mode") == "rings" else 0, trap.get("cx", 0.0), trap.get("cy", 0.0),
            trap.get("radius", 0.5), trap.get("angle", 0.0), trap.get("falloff", 2.0),
            trap.get("freq", 4.0), trap.get("strength", 1.0), phase_strength, phase_freq,
            (_lib.ITER_EXACT_WALKERS if exact_walkers else 0) | (_lib.ITER_AGGREGATE if aggregate else 0)
            | {"auto": 0, "barrier": _lib.ITER_KERNEL_BARRIER, "queue": _lib.ITER_KERNEL_QUEUE,
               "wave": _lib.ITER_KERNEL_WAVE}[kernel])
        _lib.check(_lib.lib().pyr3_iterate(self._h, C.byref(gg.c), C.byref(o)))
        self.launches += self.last_iterate_launches()

    def present_opts(self, genome: Genome, force_de_off: bool = False,
                     transparent: bool = False) -> _lib.PresentOpts:
        tm = dict(DEFAULT_TONEMAP)
        tm.update(genome.tonemap or {})
        de = genome.density
        use_de = de is not None and not force_de_off
        p = _lib.PresentOpts(
            tm["gamma"], tm["vibrancy"], tm["highlightPower"], tm["brightness"],
            tm["gammaThreshold"], 1 if use_de else 0,
            de["maxRad"] if use_de else 0.0, de["minRad"] if use_de else 0.0,
            de["curve"] if use_de else 0.0, (C.c_float * 3)(*genome.background),
            1 if transparent else 0, float(genome.scale))
        lut = bake_curves(genome.channel_curves)
        if lut is not None:  # src/visualize.ts:170-175
            p.curves_active = curves_active_mask(genome.channel_curves)
            p.curves = lut.ctypes.data
            p._curves_lut = lut  # keeps the LUT alive as long as the struct
        if genome.hsl_adjust:  # src/visualize.ts:194-198
            p.hsl_active = 1
            p.hsl_hue = genome.hsl_adjust.get("hue", 0.0)
            p.hsl_sat = genome.hsl_adjust.get("sat", 100.0) / 100.0
            p.hsl_light = genome.hsl_adjust.get("light", 0.0) / 100.0
        return p

    def present(self, genome: Genome, total_samples: int, force_de_off: bool = False,
                transparent: bool = False, out: np.ndarray | None = None,
                fmt: str = "rgba8") -> np.ndarray:
        """Density estimation + tonemap into a host RGBA image
        (src/renderer.ts:241).  fmt (FORMATS): "rgba8", "f32" (the fragment
        value), "f16" (the rgba16float texture), "png16" and "exr" (the
        png16 / exr exports of src/gpu-readback.ts:83-115, computed by the
        tonemap pass)."""
        kind, dtype = FORMATS[fmt]
        if out is None:
            out = np.zeros((self.height, self.width, 4), dtype)
        p = self.present_opts(genome, force_de_off, transparent)
        _lib.check(_lib.lib().pyr3_present(self._h, C.byref(p), int(total_samples), _lib.ptr(out), kind))
        return out

    def present_device(self, genome: Genome, total_samples: int, device_out: int,
                       force_de_off: bool = False, transparent: bool = False,
                       fmt: str = "rgba8") -> None:
        """present() into a device buffer (a pointer to W x H RGBA u8 or f32,
        e.g. a CUDA tensor's data_ptr()), queued on the renderer's stream."""
        kind = FORMATS[fmt][0]
        p = self.present_opts(genome, force_de_off, transparent)
        _lib.check(_lib.lib().pyr3_present_device(self._h, C.byref(p), int(total_samples),
                                                  C.c_void_p(int(device_out)), kind))

    def render(self, genome: Genome, seed: int = 0, **kw) -> np.ndarray:
        """reset + iterate + present (src/renderer.ts:264-278)."""
        spp = genome.quality if genome.quality is not None else DEFAULT_SPP
        w, it, samples = compute_dispatch(spp, self.width, self.height)
        self.reset(genome)
        self.iterate(genome, seed, w, it, **{k: v for k, v in kw.items() if k not in ("transparent", "force_de_off")})
        return self.present(genome, samples, kw.get("force_de_off", False), kw.get("transparent", False))

    def resize(self, width: int, height: int, oversample=None, filter_radius=None) -> None:
        os_ = max(1, int(oversample if oversample is not None else self.oversample))
        fr = filter_radius if filter_radius is not None else self.filter_radius
        o = _lib.Opts(width, height, os_, fr, self._opts.device)
        _lib.check(_lib.lib().pyr3_resize(self._h, C.byref(o)))
        self._opts = o

    def read_histogram(self):
        """(rgba u32 [superH, superW, 4], superW, superH) (src/renderer.ts:209)."""
        h = np.zeros((self.super_h, self.super_w, 4), np.uint32)
        _lib.check(_lib.lib().pyr3_read_histogram(self._h, _lib.ptr(h)))
        return h, self.super_w, self.super_h

    def read_linear(self, genome: Genome, total_samples: int) -> np.ndarray:
        """Linear scene-referred RGBA f32 [H, W, 4] of the histogram
        (src/export-linear.ts:24-47, the exr-linear export), k1 and k2 from
        deriveCalibration (src/calibration.ts:37-43) in double."""
        tm = dict(DEFAULT_TONEMAP)
        tm.update(genome.tonemap or {})
        k1 = (tm["brightness"] * 255.0 * 268.0) / 256.0
        k2 = (self.oversample ** 2 * genome.scale * genome.scale) / (255.0 * total_samples)
        out = np.zeros((self.height, self.width, 4), np.float32)
        _lib.check(_lib.lib().pyr3_read_linear(self._h, k1, k2, _lib.ptr(out)))
        return out

    def set_capture_index(self, on: bool) -> None:
        _lib.check(_lib.lib().pyr3_set_capture_index(self._h, 1 if on else 0))
        self._capture = bool(on)

    def read_index_map(self):
        idx = np.zeros((self.super_h, self.super_w), np.uint32)
        _lib.check(_lib.lib().pyr3_read_index_map(self._h, _lib.ptr(idx)))
        hist, _, _ = self.read_histogram()
        return {"idxSum": idx, "count": hist[..., 3].copy(), "width": self.super_w,
                "height": self.super_h}

    def sync(self) -> None:
        _lib.check(_lib.lib().pyr3_sync(self._h))

    def counters(self):
        s, n = C.c_uint64(), C.c_uint64()
        _lib.check(_lib.lib().pyr3_counters(self._h, C.byref(s), C.byref(n)))
        return s.value, n.value

    def last_iterate_ms(self) -> float:
        ms = C.c_float()
        _lib.check(_lib.lib().pyr3_last_iterate_ms(self._h, C.byref(ms)))
        return ms.value

    def last_iterate_launches(self) -> int:
        n = C.c_uint64()
        _lib.check(_lib.lib().pyr3_last_iterate_launches(self._h, C.byref(n)))
        return n.value

    def prepare(self, genome) -> None:
        gg = genome if isinstance(genome, GpuGenome) else GpuGenome(genome)
        _lib.check(_lib.lib().pyr3_prepare(self._h, C.byref(gg.c)))

    def destroy(self) -> None:
        if self._h:
            _lib.lib().pyr3_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def create_renderer(width: int, height: int, oversample: int = 1, filter_radius=None,
                    device: int = 0) -> Renderer:
    """createRenderer (src/renderer.ts:214)."""
    return Renderer(width, height, oversample, filter_radius, device)
