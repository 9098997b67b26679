"""Seeded synthetic workloads (the benchmark configurations).

Every genome here is generated from a fixed seed with numpy's PCG64 so the
same file can be rendered by the reference (`.pyr3.json` in
pyr3_b200/genomes/, written by `python -m pyr3_b200.workloads`).  Parameter draws follow the
configuration text:

* `plain_small()`  -- 640x480 os1 q50, 3 xforms (a..f ~ U[-1,1], weight
  ~ U[0.2,1]), {linear, sinusoidal, spherical} weights ~ U[0,1] normalised,
  colour ~ U[0,1], speed 0.5, 256 uniform-random palette entries, DE 9/0/0.4,
  gamma 4, brightness 4, vibrancy 1.  Scale = width/4, centre (0, 0).
* `headline_1080p()` -- 1920x1080 os2 q500, 12 xforms + final, post affines,
  1-4 variations per xform uniform over the whole catalog with parameters
  uniform in their documented ranges, weights Dirichlet(1), palette from
  seeded HSV stops.  DE off (the configuration sets none).
* `motion_4k()` -- 3840x2160 os2 q2000, 6 xforms mixing flam3-core and
  direct-colour variations (dc_linear / dc_perlin / dc_cylinder), 8 temporal
  samples with linearly interpolated affines, DE 15/0/0.6.
* `batch_256()` -- 256 genomes: 2-20 xforms, 1-6 catalog variations each,
  canvases from {256^2, 512^2, 800x600, 1024x768}, quality U[50, 400].
"""
from __future__ import annotations

import colorsys
import json
import os

import numpy as np

from .genome import Genome, Variation, Xform, catalog, genome_to_json, variation_index

HERE = os.path.dirname(os.path.abspath(__file__))
# flam3's original variation set (V0..V98 in the registry, pre_blur excluded).
FLAM3_CORE = [i for i in range(99) if i != 97]


def _params_for(rng: np.random.Generator, idx: int) -> list:
    entry = catalog()[idx]
    out = [0.0] * 10
    for k, rg in enumerate(entry["ranges"][:10]):
        lo, hi, _ = rg if rg else (0.0, 0.0, 0.0)
        out[k] = float(rng.uniform(lo, hi)) if hi > lo else float(lo)
    return out


def _random_affine(rng):
    return [float(v) for v in rng.uniform(-1.0, 1.0, 6)]


def _hsv_palette(rng, n_stops: int = 8):
    hs = rng.uniform(0.0, 1.0, n_stops)
    ss = rng.uniform(0.5, 1.0, n_stops)
    vs = rng.uniform(0.4, 1.0, n_stops)
    stops = []
    for k in range(n_stops):
        r, g, b = colorsys.hsv_to_rgb(hs[k], ss[k], vs[k])
        stops.append((k / (n_stops - 1), float(r), float(g), float(b)))
    return stops


def _palette_256(rgb: np.ndarray):
    return [(i / 255, float(rgb[i, 0]), float(rgb[i, 1]), float(rgb[i, 2])) for i in range(256)]


def plain_small(seed: int = 0) -> Genome:
    rng = np.random.Generator(np.random.PCG64(seed))
    names = ["linear", "sinusoidal", "spherical"]
    idxs = [variation_index(n) for n in names]
    xforms = []
    for _ in range(3):
        a, b, c, d, e, f = _random_affine(rng)
        weight = float(rng.uniform(0.2, 1.0))
        vw = rng.uniform(0.0, 1.0, 3)
        vw = vw / vw.sum()
        color = float(rng.uniform(0.0, 1.0))
        xforms.append(Xform(a=a, b=b, c=c, d=d, e=e, f=f, weight=weight, color=color,
                            color_speed=0.5,
                            variations=[Variation(i, float(w)) for i, w in zip(idxs, vw)]))
    pal = _palette_256(rng.uniform(0.0, 1.0, (256, 3)))
    width, height = 640, 480
    return Genome(name="plain-small-seed0", xforms=xforms, scale=width / 4, cx=0.0, cy=0.0,
                  palette=pal, density={"maxRad": 9.0, "minRad": 0.0, "curve": 0.4},
                  tonemap={"gamma": 4.0, "vibrancy": 1.0, "highlightPower": 1.0,
                           "brightness": 4.0, "gammaThreshold": 0.01},
                  quality=50, oversample=1, size=(width, height))


def _catalog_xform(rng, n_vars_lo: int, n_vars_hi: int, pool=None, post: bool = False,
                   weight: float = 1.0) -> Xform:
    n_all = len(catalog())
    pool = pool if pool is not None else list(range(n_all))
    nv = int(rng.integers(n_vars_lo, n_vars_hi + 1))
    vs = []
    vw = rng.uniform(0.0, 1.0, nv)
    vw = vw / vw.sum()
    for k in range(nv):
        idx = int(pool[int(rng.integers(0, len(pool)))])
        vs.append(Variation(idx, float(vw[k]), _params_for(rng, idx)))
    a, b, c, d, e, f = _random_affine(rng)
    x = Xform(a=a, b=b, c=c, d=d, e=e, f=f, weight=weight, color=float(rng.uniform(0, 1)),
              color_speed=float(rng.uniform(0.2, 0.8)), variations=vs)
    if post:
        pa, pb, pc, pd, pe, pf = (float(v) for v in rng.uniform(-0.3, 0.3, 6))
        x.post = (1.0 + pa, pb, pc, pd, 1.0 + pe, pf)
    return x


def headline_1080p(seed: int = 2) -> Genome:
    rng = np.random.Generator(np.random.PCG64(seed))
    weights = rng.dirichlet(np.ones(12))
    xforms = [_catalog_xform(rng, 1, 4, post=True, weight=float(w)) for w in weights]
    final = _catalog_xform(rng, 1, 4, post=True, weight=0.0)
    width, height = 1920, 1080
    return Genome(name="headline-1080p-12xf", xforms=xforms, finalxform=final, scale=width / 4,
                  palette=_hsv_palette(rng), quality=500, oversample=2, size=(width, height),
                  tonemap={"gamma": 4.0, "vibrancy": 1.0, "highlightPower": 1.0,
                           "brightness": 4.0, "gammaThreshold": 0.01})


def motion_4k(seed: int = 3):
    """Returns (genome at shutter open, genome at shutter close); the eight
    temporal samples interpolate the affines linearly between them."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dc = [variation_index(n) for n in ("dc_linear", "dc_perlin", "dc_cylinder")]
    xforms = []
    for k in range(6):
        pool = dc if k % 2 == 1 else FLAM3_CORE
        x = _catalog_xform(rng, 1, 2, pool=pool, weight=float(rng.uniform(0.2, 1.0)))
        if k % 2 == 1:  # give DC xforms a position-bearing variation too
            lin = variation_index("linear")
            x.variations.append(Variation(lin, 1.0))
        xforms.append(x)
    width, height = 3840, 2160
    g0 = Genome(name="motion-4k-6xf", xforms=xforms, scale=width / 4, palette=_hsv_palette(rng),
                density={"maxRad": 15.0, "minRad": 0.0, "curve": 0.6}, quality=2000,
                oversample=2, size=(width, height),
                tonemap={"gamma": 4.0, "vibrancy": 1.0, "highlightPower": 1.0,
                         "brightness": 4.0, "gammaThreshold": 0.01})
    import copy

    g1 = copy.deepcopy(g0)
    for x in g1.xforms:
        d = rng.uniform(-0.05, 0.05, 6)
        x.a, x.b, x.c, x.d, x.e, x.f = (v + float(dv) for v, dv in zip((x.a, x.b, x.c, x.d, x.e, x.f), d))
    return g0, g1


def animate_preview(seed: int = 3):
    """The motion_4k keyframes as a preview animation: 640x360, oversample
    1, 50 spp (DE radii kept); returns (g0, g1) at t = 0 and t = 1."""
    import copy

    out = []
    for g in motion_4k(seed):
        p = copy.deepcopy(g)
        p.name = "animate-preview-6xf"
        p.size = (640, 360)
        p.scale = 640 / 4
        p.oversample = 1
        p.quality = 50
        out.append(p)
    return tuple(out)


def batch_256(seed: int = 4, n: int = 256):
    rng = np.random.Generator(np.random.PCG64(seed))
    canvases = [(256, 256), (512, 512), (800, 600), (1024, 768)]
    out = []
    for k in range(n):
        nx = int(rng.integers(2, 21))
        w = rng.uniform(0.2, 1.0, nx)
        xforms = [_catalog_xform(rng, 1, 6, weight=float(wi)) for wi in w]
        cw, ch = canvases[int(rng.integers(0, 4))]
        q = float(rng.uniform(50, 400))
        out.append(Genome(name=f"batch-{k:03d}", xforms=xforms, scale=cw / 4,
                          palette=_hsv_palette(rng), quality=q, oversample=1, size=(cw, ch),
                          tonemap={"gamma": 4.0, "vibrancy": 1.0, "highlightPower": 1.0,
                                   "brightness": 4.0, "gammaThreshold": 0.01}))
    return out


def denoise_set(seed: int = 5, n: int = 72, size: int = 256, structures: int = 4):
    """Genomes for the learned denoiser: `structures` xform/variation layouts
    (4, 6, 8 and 12 xforms of 1-2 flam3-core variations each), and for every
    genome fresh affines, weights, variation weights and parameters, colours
    and palette on one of them.  Few structures keep the number of compiled
    chaos modules small; size x size canvases, oversample 1."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shapes = []
    for k in range(structures):
        nx = (4, 6, 8, 12)[k % 4]
        shapes.append([[int(FLAM3_CORE[int(rng.integers(0, len(FLAM3_CORE)))])
                        for _ in range(int(rng.integers(1, 3)))] for _ in range(nx)])
    out = []
    for i in range(n):
        sh = shapes[i % structures]
        weights = rng.dirichlet(np.ones(len(sh)))
        xforms = []
        for vars_, w in zip(sh, weights):
            vw = rng.uniform(0.2, 1.0, len(vars_))
            vw = vw / vw.sum()
            vs = [Variation(idx, float(vw[k]), _params_for(rng, idx)) for k, idx in enumerate(vars_)]
            a, b, c, d, e, f = _random_affine(rng)
            xforms.append(Xform(a=a, b=b, c=c, d=d, e=e, f=f, weight=float(w),
                                color=float(rng.uniform(0, 1)), color_speed=float(rng.uniform(0.2, 0.8)),
                                variations=vs))
        out.append(Genome(name=f"denoise-{i}", xforms=xforms, scale=size / 4, palette=_hsv_palette(rng),
                          quality=25, oversample=1, size=(size, size),
                          tonemap={"gamma": 4.0, "vibrancy": 1.0, "highlightPower": 1.0,
                                   "brightness": 4.0, "gammaThreshold": 0.01}))
    return out


def write_all(outdir: str | None = None) -> list:
    """Write the benchmark genomes as `.pyr3.json` files (the reference's v1
    schema), so the reference can render the identical genomes: the four
    single-genome configurations (motion_4k and animate_preview as their
    two keyframes) and the eight batch_256 genomes the parity tests render
    (the generator reproduces the other 248 from the same seed)."""
    outdir = outdir or os.path.join(HERE, "genomes")
    os.makedirs(outdir, exist_ok=True)
    items = {"plain_small.pyr3.json": plain_small(), "headline_1080p.pyr3.json": headline_1080p()}
    g0, g1 = motion_4k()
    items["motion_4k_open.pyr3.json"] = g0
    items["motion_4k_close.pyr3.json"] = g1
    a0, a1 = animate_preview()
    items["animate_preview_open.pyr3.json"] = a0
    items["animate_preview_close.pyr3.json"] = a1
    for g in batch_256()[:8]:
        items[f"{g.name}.pyr3.json"] = g
    paths = []
    for name, g in items.items():
        path = os.path.join(outdir, name)
        with open(path, "w") as f:
            json.dump(genome_to_json(g), f, indent=1)
            f.write("\n")
        paths.append(path)
    return paths


if __name__ == "__main__":
    for p in write_all():
        print(p)
