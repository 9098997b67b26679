"""Motion-blurred frames: N temporal sub-frames accumulated into one histogram.

Restates the host side of the reference's animation render for one output
frame:

* ``temporal_filter``   -- createTemporalFilter (src/temporal-filter.ts:25-77),
  itself flam3's flam3_create_temporal_filter: sub-frame time offsets and
  weights (box / gaussian / exp), normalised so the largest weight is 1;
* ``apportion_walkers`` -- apportionWalkers (src/animate-render.ts:27-41):
  largest-remainder (Hamilton) split of an integer walker budget;
* ``interpolate_linear`` -- the linear two-keyframe blend of interpolate()
  (src/interpolate.ts:58-260, affine part :469-475 and blend :1229):
  every numeric xform field is c0 * v0 + c1 * v1 with
  c0 = (t1 - time) / (t1 - t0), c1 = 1 - c0;
* ``render_motion_frame`` -- renderAnimationFrame (src/animate-render.ts:73-176):
  reset with the centre-time genome, one iterate per sub-frame at
  time + delta[i] with walkers apportioned by filter weight and seed
  (base + i * 0x9e3779b1) mod 2^32, then a single present with the total
  sample count;
* ``AnimationBatch`` -- the frame loop of bin/pyr3-animate.ts (frame k at
  time k / fps, each through renderAnimationFrame) for many frames at once:
  every frame's sub-frames go into one pyr3_batch, each frame accumulating
  into its own renderer, so a sequence of frames too small to fill the GPU
  one by one runs as one graph launch.

The keyframe blend covers keyframes of the same structure (same xform
count and variation lists), which is what a motion-blurred frame of one
animated genome needs; the reference's xform alignment, easing curves,
Catmull-Rom and log-polar affine modes belong to its animation editor and
are not restated here.
"""
from __future__ import annotations

import copy
import ctypes as C
import math

from . import _lib
from .genome import Genome, Xform
from .renderer import DEFAULT_WALKER_JITTER, GpuGenome, Renderer, compute_dispatch

GOLDEN = 0x9E3779B1  # per-sub-frame seed stride (src/animate-render.ts:151)


def temporal_filter(numsteps: int, kind: str = "box", width: float = 1.0, exp: float = 0.0):
    """(deltas, filter, sumfilt) for `numsteps` sub-frames
    (src/temporal-filter.ts:25-77)."""
    if numsteps <= 1:
        return [0.0], [1.0], 1.0
    deltas = [(i / (numsteps - 1) - 0.5) * width for i in range(numsteps)]
    if kind == "exp":
        filt = [(((i + 1) / numsteps) if exp >= 0 else ((numsteps - i) / numsteps)) ** abs(exp)
                for i in range(numsteps)]
    elif kind == "gaussian":
        half = numsteps / 2.0
        support = 1.5  # flam3's gaussian spatial support
        filt = [math.exp(-2.0 * ((support * abs(i - half)) / half) ** 2) * math.sqrt(2.0 / math.pi)
                for i in range(numsteps)]
    else:
        filt = [1.0] * numsteps
    mx = max(filt)
    filt = [v / mx for v in filt]
    return deltas, filt, sum(filt) / numsteps


def apportion_walkers(total: int, weights) -> list:
    """Largest-remainder split of `total` walkers by `weights`; sums exactly
    to `total`, zero-weight entries get 0 (src/animate-render.ts:27-41)."""
    n = len(weights)
    if n == 0:
        return []
    sum_w = sum(w for w in weights if w > 0)
    if sum_w <= 0 or total <= 0:
        return [0] * n
    quotas = [total * max(0.0, w) / sum_w for w in weights]
    out = [math.floor(q) for q in quotas]
    deficit = total - sum(out)
    order = sorted(range(n), key=lambda i: -(quotas[i] - math.floor(quotas[i])))  # stable
    for k in range(min(deficit, n)):
        out[order[k]] += 1
    return out


def _blend(v0, v1, c0, c1):
    return c0 * v0 + c1 * v1


def _blend_xform(x0: Xform, x1: Xform, c0: float, c1: float) -> Xform:
    if len(x0.variations) != len(x1.variations) or any(
            a.index != b.index for a, b in zip(x0.variations, x1.variations)):
        raise ValueError("keyframes differ in structure (variation lists)")
    x = copy.deepcopy(x0)
    for k in ("a", "b", "c", "d", "e", "f", "weight", "color", "color_speed"):
        setattr(x, k, _blend(getattr(x0, k), getattr(x1, k), c0, c1))
    if x0.opacity is not None and x1.opacity is not None:
        x.opacity = _blend(x0.opacity, x1.opacity, c0, c1)
    if x0.post is not None and x1.post is not None:
        x.post = tuple(_blend(p, q, c0, c1) for p, q in zip(x0.post, x1.post))
    for v, v0, v1 in zip(x.variations, x0.variations, x1.variations):
        v.weight = _blend(v0.weight, v1.weight, c0, c1)
        v.params = [_blend(p, q, c0, c1) for p, q in zip(v0.params, v1.params)]
    return x


def interpolate_linear(g0: Genome, g1: Genome, time: float, t0: float = 0.0,
                       t1: float = 1.0) -> Genome:
    """Genome at `time` between keyframes g0 (at t0) and g1 (at t1), blended
    linearly; extrapolates outside [t0, t1] as the reference does."""
    if len(g0.xforms) != len(g1.xforms) or (g0.finalxform is None) != (g1.finalxform is None):
        raise ValueError("keyframes differ in structure (xform count / final xform)")
    c0 = (t1 - time) / (t1 - t0)
    c1 = 1.0 - c0
    g = copy.deepcopy(g0)
    g.xforms = [_blend_xform(a, b, c0, c1) for a, b in zip(g0.xforms, g1.xforms)]
    if g0.finalxform is not None:
        g.finalxform = _blend_xform(g0.finalxform, g1.finalxform, c0, c1)
    for k in ("scale", "cx", "cy", "rotate"):
        setattr(g, k, _blend(getattr(g0, k), getattr(g1, k), c0, c1))
    return g


def render_motion_frame(renderer: Renderer, g0: Genome, g1: Genome, time: float = 0.5,
                        ntemporal: int = 8, filter_kind: str = "box", filter_width: float = 1.0,
                        filter_exp: float = 0.0, seed: int = 0, **iterate_kw):
    """One motion-blurred frame (src/animate-render.ts:73-176).  Returns
    (total_samples, walkers per sub-frame); the image is left for
    renderer.present(centre genome, total_samples)."""
    centre = interpolate_linear(g0, g1, time)
    walkers, iters, _ = compute_dispatch(centre.quality or 16, renderer.width, renderer.height)
    renderer.reset(centre)
    n = max(1, int(ntemporal))
    if n == 1:
        renderer.iterate(centre, seed & 0xFFFFFFFF, walkers, iters, **iterate_kw)
        return walkers * iters, [walkers]
    deltas, filt, _ = temporal_filter(n, filter_kind, filter_width, filter_exp)
    counts = apportion_walkers(walkers, filt)
    total = 0
    for i, w in enumerate(counts):
        if w == 0:
            continue
        sub = interpolate_linear(g0, g1, time + deltas[i])
        renderer.iterate(sub, (seed + i * GOLDEN) & 0xFFFFFFFF, w, iters, **iterate_kw)
        total += w
    return total * iters, counts


def _frame_plan(g0: Genome, g1: Genome, time: float, width: int, height: int, ntemporal: int,
                filter_kind: str, filter_width: float, filter_exp: float, seed: int):
    """renderAnimationFrame's plan for one frame: (centre genome, iterate
    requests [(genome, seed, walkers, iters)], total samples)."""
    centre = interpolate_linear(g0, g1, time)
    walkers, iters, _ = compute_dispatch(centre.quality or 16, width, height)
    n = max(1, int(ntemporal))
    if n == 1:
        return centre, [(centre, seed & 0xFFFFFFFF, walkers, iters)], walkers * iters
    deltas, filt, _ = temporal_filter(n, filter_kind, filter_width, filter_exp)
    reqs = [(interpolate_linear(g0, g1, time + deltas[i]), (seed + i * GOLDEN) & 0xFFFFFFFF, w, iters)
            for i, w in enumerate(apportion_walkers(walkers, filt)) if w > 0]
    return centre, reqs, sum(r[2] for r in reqs) * iters


class AnimationBatch:
    """Frames at `times` of the two-keyframe animation g0 -> g1, rendered
    together: frame k is renderAnimationFrame (src/animate-render.ts:73-176)
    at times[k] -- its renderer reset with the centre genome, one iterate
    per sub-frame -- and every sub-frame of every frame is one genome of a
    single pyr3_batch, whose frames share nothing but the GPU.  run() clears
    the frames' histograms and accumulates all of them; present(k) returns
    frame k.  Sizes default to g0's; seed is every frame's base seed, as
    bin/pyr3-animate.ts passes one seed to all frames.

        ab = AnimationBatch(g0, g1, [k / 30 for k in range(30)], ntemporal=8)
        ab.run(); ab.sync()
        frames = [ab.present(k) for k in range(30)]
    """

    def __init__(self, g0: Genome, g1: Genome, times, width: int | None = None,
                 height: int | None = None, oversample: int | None = None, ntemporal: int = 8,
                 filter_kind: str = "box", filter_width: float = 1.0, filter_exp: float = 0.0,
                 seed: int = 0, n_streams: int = 64, device: int = 0):
        W = width or (g0.size[0] if g0.size else 1024)
        H = height or (g0.size[1] if g0.size else 1024)
        os_ = oversample or g0.oversample or 1
        self.renderers, self.centres, self.samples = [], [], []
        self._keep = []
        entries = []
        for t in times:
            centre, reqs, total = _frame_plan(g0, g1, float(t), W, H, ntemporal, filter_kind,
                                              filter_width, filter_exp, seed)
            r = Renderer(W, H, os_, g0.filter_radius, device=device)
            r.reset(centre)
            self.renderers.append(r)
            self.centres.append(centre)
            self.samples.append(total)
            entries += [(r, req) for req in reqs]
        n = len(entries)
        opts = (_lib.IterateOpts * n)()
        gcs = (_lib.GenomeC * n)()
        hs = (C.c_void_p * n)()
        for i, (r, (g, sd, w, it)) in enumerate(entries):
            gg = GpuGenome(g)
            self._keep.append(gg)
            o = opts[i]
            o.walkers, o.iters_per_walker, o.seed = w, it, sd
            o.walker_jitter = DEFAULT_WALKER_JITTER
            o.flow_strength = o.trap_strength = o.phase_strength = o.phase_freq = 1.0
            gcs[i] = gg.c
            hs[i] = r.handle.value
        self.n_genomes = n
        self._opts, self._gcs, self._hs = opts, gcs, hs
        self._b = C.c_void_p()
        _lib.check(_lib.lib().pyr3_batch_create(hs, gcs, opts, n, n_streams, C.byref(self._b)))

    def run(self) -> None:
        """Clear every frame's histogram and accumulate all sub-frames."""
        _lib.check(_lib.lib().pyr3_batch_run(self._b))

    def sync(self):
        """Wait for the last run; (device ms, total samples)."""
        ms, s = C.c_float(), C.c_uint64()
        _lib.check(_lib.lib().pyr3_batch_sync(self._b, C.byref(ms), C.byref(s)))
        return ms.value, s.value

    def present(self, k: int, **kw):
        """Frame k: present of the centre genome with the frame's samples."""
        return self.renderers[k].present(self.centres[k], self.samples[k], **kw)

    def destroy(self) -> None:
        if self._b:
            _lib.lib().pyr3_batch_destroy(self._b)
            self._b = C.c_void_p()
        for r in self.renderers:
            r.destroy()
        self.renderers = []

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
