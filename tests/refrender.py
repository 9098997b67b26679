"""Whole renders by the reference's own chaos loop (chaos_main of
src/shaders/chaos.wgsl, translated for the CPU in oracle/_ref) for the GPU
parity tests: the uniform block of src/chaos.ts:381-456 filled from a
genome, the final-xform slot (src/genome.ts:432), the weight x xaos pick
table (src/genome.ts:482-534), and the walker streams of packIsaacStates
(src/isaac.ts:194-229).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import math
import os

import numpy as np

from oracle import oracle as O
from pyr3_b200 import genome as G

THREADS = max(1, os.cpu_count() or 1)

# (gamma, vibrancy, highlight power, background, transparent): the
# reference's DEFAULT_TONEMAP (src/tonemap.ts:31-37: gamma 2.4, vibrancy 0),
# the C1 point (gamma 4, vibrancy 1) and the branches of calc_newrgb
# (visualize_u32.wgsl:96-145: highpow below / above 1), the vibrancy blend
# near 1, a non-black background and transparent output.
TONEMAP_CASES = [
    (2.4, 0.0, 1.0, (0.0, 0.0, 0.0), False),
    (2.4, 0.0, 1.0, (0.1, 0.2, 0.3), True),
    (4.0, 1.0, 1.0, (0.0, 0.0, 0.0), False),
    (4.0, 0.5, 0.3, (0.2, 0.05, 0.4), False),
    (4.0, 0.5, 2.0, (0.0, 0.0, 0.0), True),
    (0.8, 1.0, 2.0, (0.3, 0.3, 0.3), False),
    (0.8, 0.0, 0.3, (0.0, 0.0, 0.0), True),
    (2.4, 1.0, 0.3, (0.05, 0.1, 0.0), True),
    (4.0, 0.999, 1.0, (0.0, 0.0, 0.0), False),
]


def uniforms(g, super_w, super_h, iters, walkers, seed, oversample=1, slots=None):
    """The reference's 31-slot chaos uniform block for genome g (already
    expanded for the GPU) on a super_w x super_h histogram."""
    u = np.zeros(31, np.uint32)
    f = u.view(np.float32)
    i32 = u.view(np.int32)
    u[0], u[1], u[2], u[3] = super_w, super_h, iters, 200
    f[4] = np.float32(g.scale * oversample)
    f[5], f[6] = g.cx, g.cy
    u[7] = seed & 0xFFFFFFFF
    i32[8] = G.final_slot(g)
    f[9] = np.float32((g.rotate or 0.0) * math.pi / 180.0)
    u[10] = 1 if g.palette_mode == "linear" else 0
    u[12] = walkers
    f[13] = np.float32(1e-7)
    # render-time colour defaults (src/chaos.ts:421-456), all inactive
    f[16], f[17], f[22], f[24], f[25], f[26], f[27], f[28], f[29] = 1.0, 2.0, 0.5, 1.0, 2.0, 4.0, 1.0, 1.0, 1.0
    f[30] = np.float32(min(1.0, max(0.0, g.xform_blend or 0.0)))
    for k, (t, v) in (slots or {}).items():
        if t == "u":
            u[k] = v
        else:
            f[k] = v
    return u


def chaos(g, super_w, super_h, iters, walkers, seed, oversample=1, slots=None, hist=None,
          walker0=0, threads=THREADS):
    """Accumulate walkers [walker0, walker0 + walkers) x iters post-fuse
    samples of genome g into hist (u32, super_w x super_h x 4) with the
    reference's chaos_main; returns hist."""
    gg = G.expand_for_gpu(g)
    if hist is None:
        hist = np.zeros(super_w * super_h * 4, np.uint32)
    u = uniforms(gg, super_w, super_h, iters, walker0 + walkers, seed, oversample, slots)
    xa = G.xaos_matrix(gg)
    distrib = O.pack_xform_distrib([x.weight for x in gg.xforms],
                                   None if xa is None else xa.astype(np.float64))
    pal = G.bake_lut(gg.palette, gg.palette_hue, gg.palette_interp)
    isaac = O.pack_isaac_states(walker0 + walkers, seed)
    O.ref_chaos_run(u, G.pack_xforms(gg), len(gg.xforms), pal, distrib, isaac, walker0,
                    walker0 + walkers, hist, threads)
    return hist


def collapse_counts(hist, width, height, oversample):
    """Count channel summed over each output pixel's oversample block."""
    h = np.asarray(hist).reshape(height * oversample, width * oversample, 4)[..., 3].astype(np.float64)
    return h.reshape(height, oversample, width, oversample).sum(axis=(1, 3))


def log_density_l1(a, b, width, height, oversample):
    """Relative L1 of log1p(count / 255) per output pixel, against b."""
    la = np.log1p(collapse_counts(a, width, height, oversample) / 255.0)
    lb = np.log1p(collapse_counts(b, width, height, oversample) / 255.0)
    return float(np.abs(la - lb).sum() / lb.sum())


def psnr(x, y):
    mse = float(((np.asarray(x, np.float64) - np.asarray(y, np.float64)) ** 2).mean())
    return 10.0 * np.log10(1.0 / max(mse, 1e-20))
