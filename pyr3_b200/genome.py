"""Genome model and GPU packers (host side of the reference's chaos pass).

Mirrors the reference's data model and the packing that feeds its chaos
kernel, so a genome means the same thing here:

* `Genome` / `Xform` / `Variation` follow src/genome.ts:19-168 and
  src/variations.ts:745-778; `genome_from_json` reads the `.pyr3.json` v1
  schema of src/serialize.ts:14-126 (the fields the render path uses).
* `pack_xforms` writes the 116-float record per xform of
  src/genome.ts:293-421 (affine0 [a,b,c,w], affine1 [d,e,f,nvars],
  colour [color, speed, opacity, dc_flag], post0/post1, vars[8],
  vars_extra[8], vars_extra2[8]); `final_slot` is src/genome.ts:432.
* `expand_for_gpu` is expandGenomeForGPU (src/symmetry.ts:21-90): inactive
  xforms/variations get weight 0 and symmetry becomes explicit xforms.
* `bake_lut` is bakeLUT (src/palette.ts:71-125), 256 x RGBA f32, alpha 0.
"""
from __future__ import annotations

import copy
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

XFORM_FLOATS = 116
MAX_XFORMS = 128
MAX_VARS = 8

_CAT = None


def catalog() -> dict:
    """Variation catalog: index, name, positional parameter names, defaults,
    documented ranges, direct-colour flag (extracted from the reference)."""
    global _CAT
    if _CAT is None:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "catalog.json")) as f:
            _CAT = json.load(f)["variations"]
    return _CAT


def variation_index(name: str) -> int:
    for v in catalog():
        if v["name"] == name:
            return v["idx"]
    raise KeyError(f"unknown variation {name!r}")


@dataclass
class Variation:
    index: int
    weight: float
    params: list = field(default_factory=lambda: [0.0] * 10)  # param0..param9
    active: bool = True


@dataclass
class Xform:
    a: float = 1.0
    b: float = 0.0
    c: float = 0.0
    d: float = 0.0
    e: float = 1.0
    f: float = 0.0
    weight: float = 1.0
    color: float = 0.0
    color_speed: float = 0.5
    variations: list = field(default_factory=list)
    opacity: float | None = None
    xaos: list | None = None
    post: tuple | None = None  # (a, b, c, d, e, f)
    active: bool = True


@dataclass
class Genome:
    name: str = "genome"
    xforms: list = field(default_factory=list)
    scale: float = 100.0
    cx: float = 0.0
    cy: float = 0.0
    palette: list = field(default_factory=list)  # stops: (t, r, g, b)
    palette_hue: float = 0.0
    palette_interp: str = "linear"  # bakeLUT mode: linear | step | smooth
    finalxform: Xform | None = None
    symmetry: tuple | None = None  # ("rotational"|"dihedral", n)
    density: dict | None = None  # {maxRad, minRad, curve}
    tonemap: dict | None = None  # {gamma, vibrancy, highlightPower, brightness, gammaThreshold}
    rotate: float = 0.0
    xform_blend: float = 0.0
    quality: float | None = None
    oversample: int = 1
    size: tuple | None = None  # (width, height)
    filter_radius: float | None = None
    background: tuple = (0.0, 0.0, 0.0)
    palette_mode: str = "step"  # splat-time palette sampling: step | linear
    channel_curves: dict | None = None  # {composite, r, g, b, luma: [(x, y), ...]}
    hsl_adjust: dict | None = None  # {hue (degrees), sat (percent), light (percent)}


DEFAULT_TONEMAP = {"gamma": 2.4, "vibrancy": 0.0, "highlightPower": 1.0, "brightness": 1.0,
                   "gammaThreshold": 0.01}  # src/tonemap.ts:31-37


# ------------------------------------------------------------------ JSON
def _xform_from_json(j: dict, final: bool) -> Xform:
    cat = catalog()
    by_name = {v["name"]: v for v in cat}
    af = j["affine"]
    vs = []
    for vj in j.get("variations", []):
        entry = by_name.get(vj["name"])
        if entry is None:
            raise ValueError(f"unknown variation {vj['name']!r}")
        params = list(entry["defaults"]) + [0.0] * (10 - len(entry["defaults"]))
        for k, pname in enumerate(entry["params"][:10]):
            if "params" in vj and pname in vj["params"]:
                params[k] = float(vj["params"][pname])
        vs.append(Variation(entry["idx"], float(vj["weight"]), params, vj.get("active", True)))
    post = j.get("post")
    return Xform(a=af["a"], b=af["b"], c=af["c"], d=af["d"], e=af["e"], f=af["f"],
                 weight=0.0 if final else float(j["weight"]), color=float(j["color"]),
                 color_speed=float(j["colorSpeed"]), variations=vs, opacity=j.get("opacity"),
                 xaos=j.get("xaos"),
                 post=(post["a"], post["b"], post["c"], post["d"], post["e"], post["f"]) if post else None,
                 active=j.get("active", True))


def genome_from_json(j) -> Genome:
    """Parse a `.pyr3.json` v1 payload (src/serialize.ts:1040)."""
    if isinstance(j, (str, bytes)):
        j = json.loads(j)
    if j.get("version") != 1:
        raise ValueError("only .pyr3.json version 1 is supported")
    vp = j["viewport"]
    pal = j["palette"]
    g = Genome(name=j.get("name", "genome"), scale=float(vp["scale"]), cx=float(vp["cx"]),
               cy=float(vp["cy"]),
               palette=[(s["t"], s["r"], s["g"], s["b"]) for s in pal["stops"]],
               palette_hue=float(pal.get("hue", 0.0)), palette_interp=pal.get("mode", "linear"))
    g.xforms = [_xform_from_json(x, False) for x in j["xforms"]]
    if j.get("finalxform"):
        g.finalxform = _xform_from_json(j["finalxform"], True)
    if j.get("symmetry"):
        g.symmetry = (j["symmetry"]["kind"], int(j["symmetry"]["n"]))
    g.density = j.get("density")
    g.tonemap = j.get("tonemap")
    g.rotate = float(j.get("rotate", 0.0))
    g.xform_blend = float(j.get("xformBlend", 0.0))
    g.quality = j.get("quality")
    g.oversample = int(j.get("oversample", 1))
    if j.get("size"):
        g.size = (int(j["size"]["width"]), int(j["size"]["height"]))
    if j.get("spatialFilter"):
        g.filter_radius = float(j["spatialFilter"]["radius"])
    if j.get("background"):
        g.background = tuple(float(c) for c in j["background"])
    g.palette_mode = j.get("paletteMode", "step")
    if j.get("channelCurves"):
        g.channel_curves = {ch: [(float(p["x"]), float(p["y"])) for p in pts]
                            for ch, pts in j["channelCurves"].items()}
    if j.get("hslAdjust"):
        g.hsl_adjust = {k: float(v) for k, v in j["hslAdjust"].items()}
    return g


def _xform_to_json(x: Xform, final: bool) -> dict:
    cat = catalog()
    out = {"color": x.color, "colorSpeed": x.color_speed,
           "affine": {"a": x.a, "b": x.b, "c": x.c, "d": x.d, "e": x.e, "f": x.f},
           "variations": []}
    if not final:
        out["weight"] = x.weight
    for v in x.variations:
        entry = cat[v.index]
        vj = {"name": entry["name"], "weight": v.weight}
        if entry["params"]:
            vj["params"] = {p: float(v.params[k]) for k, p in enumerate(entry["params"][:10])}
        if not v.active:
            vj["active"] = False
        out["variations"].append(vj)
    if x.opacity is not None and x.opacity != 1.0:
        out["opacity"] = x.opacity
    if x.xaos is not None:
        out["xaos"] = list(x.xaos)
    if x.post is not None:
        out["post"] = dict(zip("abcdef", x.post))
    if not x.active:
        out["active"] = False
    return out


def genome_to_json(g: Genome) -> dict:
    """Serialise to the `.pyr3.json` v1 schema (src/serialize.ts:878)."""
    j = {"version": 1, "name": g.name, "viewport": {"scale": g.scale, "cx": g.cx, "cy": g.cy},
         "palette": {"name": g.name + "-palette",
                     "stops": [{"t": t, "r": r, "g": gg, "b": b} for t, r, gg, b in g.palette]},
         "xforms": [_xform_to_json(x, False) for x in g.xforms]}
    if g.palette_interp != "linear":
        j["palette"]["mode"] = g.palette_interp
    if g.palette_hue:
        j["palette"]["hue"] = g.palette_hue
    if g.finalxform is not None:
        j["finalxform"] = _xform_to_json(g.finalxform, True)
    if g.symmetry:
        j["symmetry"] = {"kind": g.symmetry[0], "n": g.symmetry[1]}
    for key, val in (("density", g.density), ("tonemap", g.tonemap), ("quality", g.quality)):
        if val is not None:
            j[key] = val
    if g.rotate:
        j["rotate"] = g.rotate
    if g.xform_blend:
        j["xformBlend"] = g.xform_blend
    if g.oversample != 1:
        j["oversample"] = g.oversample
    if g.size:
        j["size"] = {"width": g.size[0], "height": g.size[1]}
    if g.filter_radius is not None:
        j["spatialFilter"] = {"radius": g.filter_radius, "shape": "gaussian"}
    if any(g.background):
        j["background"] = list(g.background)
    if g.palette_mode != "step":
        j["paletteMode"] = g.palette_mode
    return j


# -------------------------------------------------------- symmetry + active
def _round6(x: float) -> float:
    return math.floor(x * 1e6 + 0.5) / 1e6  # JS Math.round(x * 1e6) / 1e6


def symmetry_xforms(kind: str, n: int) -> list:
    """generateSymmetryXforms (src/symmetry.ts:92-117)."""
    out = []
    if kind == "rotational" and n == 1:
        return out
    lin = variation_index("linear")

    def op(a, b, d, e, color):
        return Xform(a=a, b=b, c=0.0, d=d, e=e, f=0.0, weight=1.0, color=color, color_speed=0.0,
                     variations=[Variation(lin, 1.0)])

    if kind == "dihedral":
        out.append(op(-1.0, 0.0, 0.0, 1.0, 1.0))
    ang = (2 * math.pi) / n
    for k in range(1, n):
        c = _round6(math.cos(k * ang))
        s = _round6(math.sin(k * ang))
        color = 0.0 if n < 3 else (k - 1) / (n - 2)
        out.append(op(c, -s, s, c, color))
    return out


def expand_for_gpu(g: Genome) -> Genome:
    """expandGenomeForGPU (src/symmetry.ts:21-46)."""
    need = any((not x.active) or any(not v.active for v in x.variations) for x in g.xforms)
    out = g
    if need:
        out = copy.deepcopy(g)
        for x in out.xforms:
            if not x.active:
                x.weight = 0.0
            for v in x.variations:
                if not v.active:
                    v.weight = 0.0
    if out.symmetry:
        extras = symmetry_xforms(*out.symmetry)
        if extras:
            if len(out.xforms) + len(extras) > MAX_XFORMS:
                raise ValueError("symmetry expansion exceeds MAX_XFORMS (128)")
            if out is g:
                out = copy.deepcopy(g)
            out.xforms = out.xforms + extras
            out.symmetry = None
    return out


# ------------------------------------------------------------------ packers
def _pack_one(buf: np.ndarray, slot: int, x: Xform) -> None:
    o = slot * XFORM_FLOATS
    n = min(len(x.variations), MAX_VARS)
    buf[o + 0:o + 4] = (x.a, x.b, x.c, x.weight)
    buf[o + 4:o + 8] = (x.d, x.e, x.f, n)
    buf[o + 8] = x.color
    buf[o + 9] = x.color_speed
    buf[o + 10] = max(0.0, min(1.0, 1.0 if x.opacity is None else x.opacity))
    dcset = {v["idx"] for v in catalog() if v["dc"]}
    buf[o + 11] = 1.0 if any(v.active and v.index in dcset for v in x.variations) else 0.0
    if x.post is not None:
        pa, pb, pc, pd, pe, pf = x.post
        buf[o + 12:o + 16] = (pa, pb, pc, 1.0)
        buf[o + 16:o + 19] = (pd, pe, pf)
    for k in range(n):
        v = x.variations[k]
        p = list(v.params) + [0.0] * (10 - len(v.params))
        vo = o + 20 + 4 * k
        buf[vo:vo + 4] = (v.index, v.weight, p[0], p[1])
        ve = o + 52 + 4 * k
        buf[ve:ve + 4] = p[2:6]
        ve2 = o + 84 + 4 * k
        buf[ve2:ve2 + 4] = p[6:10]


def pack_xforms(g: Genome) -> np.ndarray:
    """packXforms (src/genome.ts:408-421): f32 records, final xform last."""
    total = len(g.xforms) + (1 if g.finalxform is not None else 0)
    buf = np.zeros(total * XFORM_FLOATS, np.float32)
    for i, x in enumerate(g.xforms):
        _pack_one(buf, i, x)
    if g.finalxform is not None:
        _pack_one(buf, len(g.xforms), g.finalxform)
    return buf


def final_slot(g: Genome) -> int:
    """finalXformSlot (src/genome.ts:432)."""
    return len(g.xforms) if (g.finalxform is not None and g.finalxform.active) else -1


def xaos_matrix(g: Genome) -> np.ndarray | None:
    """Dense xaos[prev][next] with missing entries = 1.0 (src/genome.ts:498)."""
    if not any(x.xaos for x in g.xforms):
        return None
    n = len(g.xforms)
    m = np.ones((n, n), np.float32)
    for i, x in enumerate(g.xforms):
        if x.xaos:
            for j, v in enumerate(x.xaos[:n]):
                m[i, j] = v
    return m


def _catmull(u, xa, xb, xc, xd):
    B = 0.5
    c = u * u * u * (-B * xa + (2 - B) * xb + (B - 2) * xc + B * xd)
    c += u * u * (2 * B * xa + (B - 3) * xb + (3 - 2 * B) * xc - B * xd)
    c += u * (-B * xa + B * xc)
    return c + xb


def _rotate_hue(r, g, b, hue):
    """rotateHueRGB (src/palette.ts:130) via rgbToHsv / hsvToRgb
    (src/color-math.ts:2-26); JS `%` keeps the dividend's sign (math.fmod)."""
    mx, mn = max(r, g, b), min(r, g, b)
    d = mx - mn
    v, s, h = mx, (0.0 if mx == 0 else d / mx), 0.0
    if d != 0:
        if mx == r:
            h = math.fmod((g - b) / d, 6)
        elif mx == g:
            h = (b - r) / d + 2
        else:
            h = (r - g) / d + 4
        h *= 60
        if h < 0:
            h += 360
    h = math.fmod(math.fmod(h + hue, 360) + 360, 360)
    c = v * s
    x = c * (1 - abs(math.fmod(h / 60, 2) - 1))
    m = v - c
    rp = gp = bp = 0.0
    if h < 60:
        rp, gp = c, x
    elif h < 120:
        rp, gp = x, c
    elif h < 180:
        gp, bp = c, x
    elif h < 240:
        gp, bp = x, c
    elif h < 300:
        rp, bp = x, c
    else:
        rp, bp = c, x
    return rp + m, gp + m, bp + m


def bake_lut(stops, hue: float = 0.0, mode: str = "linear") -> np.ndarray:
    """bakeLUT (src/palette.ts:71-125): 256 x RGBA f32 (alpha 0)."""
    st = [(t, *_rotate_hue(r, g, b, hue)) if hue else (t, r, g, b) for t, r, g, b in stops]
    st = sorted(st, key=lambda s: s[0])
    out = np.zeros(1024, np.float32)
    ns = len(st)
    for i in range(256):
        t = i / 255
        lo, hi = 0, ns - 1
        for s in range(ns - 1):
            if st[s][0] <= t <= st[s + 1][0]:
                lo, hi = s, s + 1
                break
        L, H = st[lo], st[hi]
        if mode == "step":
            rgb = L[1:]
        else:
            span = (H[0] - L[0]) or 1
            u = max(0.0, min(1.0, (t - L[0]) / span))
            if mode == "smooth" and ns >= 3:
                A = st[max(0, lo - 1)]
                D = st[min(ns - 1, hi + 1)]
                rgb = [max(0.0, min(1.0, _catmull(u, A[c], L[c], H[c], D[c]))) for c in (1, 2, 3)]
            else:
                rgb = [L[c] + (H[c] - L[c]) * u for c in (1, 2, 3)]
        out[i * 4:i * 4 + 3] = rgb
    return out


# ------------------------------------------------------------ colour curves
# src/channel-curves.ts: five 256-entry LUTs (composite, r, g, b, luma) and
# the bit mask of the channels that are not the identity.
CURVE_CHANNELS = ("composite", "r", "g", "b", "luma")


def _curve_is_identity(pts) -> bool:
    return len(pts) == 2 and tuple(pts[0]) == (0, 0) and tuple(pts[1]) == (1, 1)


def curves_active_mask(curves) -> int:
    """channel-curves.ts activeMask: bit i set when channel i is not identity."""
    if not curves:
        return 0
    return sum(1 << i for i, ch in enumerate(CURVE_CHANNELS)
               if not _curve_is_identity(curves.get(ch, [(0, 0), (1, 1)])))


def eval_curve(pts, x: float) -> float:
    """Catmull-Rom (B = 0.5) through the control points with duplicated
    end neighbours, clamped to the end values (channel-curves.ts evalCurve)."""
    first, last = pts[0], pts[-1]
    if x <= first[0]:
        return first[1]
    if x >= last[0]:
        return last[1]
    if len(pts) < 3:
        dx = pts[1][0] - first[0]
        if dx < 1e-9:
            return first[1]
        return first[1] + (x - first[0]) / dx * (pts[1][1] - first[1])
    i = 0
    while i < len(pts) - 1 and pts[i + 1][0] < x:
        i += 1
    xa, xb = pts[max(0, i - 1)][1], pts[i][1]
    xc, xd = pts[i + 1][1], pts[min(len(pts) - 1, i + 2)][1]
    seg = pts[i + 1][0] - pts[i][0]
    if seg < 1e-9:
        return xb
    u = (x - pts[i][0]) / seg
    bb = 0.5
    c = u * u * u * (-bb * xa + (2 - bb) * xb + (bb - 2) * xc + bb * xd)
    c += u * u * (2 * bb * xa + (bb - 3) * xb + (3 - 2 * bb) * xc - bb * xd)
    c += u * (-bb * xa + bb * xc)
    return c + xb


def bake_curves(curves) -> np.ndarray | None:
    """5 x 256 f32 LUT (channel-curves.ts bakeCurves), None when every
    channel is the identity."""
    if curves_active_mask(curves) == 0:
        return None
    out = np.zeros(5 * 256, np.float32)
    for ch, name in enumerate(CURVE_CHANNELS):
        pts = curves.get(name, [(0, 0), (1, 1)])
        for i in range(256):
            out[ch * 256 + i] = min(1.0, max(0.0, eval_curve(pts, i / 255)))
    return out
