"""Regenerate pyr3_b200/catalog.json from the reference's variation registry.

The catalog is the genome-format contract: each variation's stable index and
name (src/variations.ts `V`, lines 24-643), its positional parameter names
(src/serialize.ts `VARIATION_PARAMS`, lines 127-473), the file-format
defaults for omitted parameters (src/serialize.ts `VARIATION_DEFAULTS`,
lines 487-504), the documented parameter ranges (src/variation-catalog-data.ts
`ParamDoc{default,min,max}`), and the direct-colour set
(src/variations.ts `DC_VARIATION_SET`, lines 681-692).  These tables have to
match the reference exactly for genome files to mean the same thing, so they
are extracted, not rewritten.  Run in a checkout that has the reference:

    python -m pyr3_b200.catalog_gen [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import math
import os
import re
import sys


def _block(text: str, start_pat: str) -> str:
    i = text.index(start_pat)
    j = text.index("\n}", i)
    return text[i:j]


def _num(expr: str) -> float:
    """Evaluate a numeric TS literal such as `-Math.PI / 4` or `1e-3`."""
    e = expr.strip().replace("Math.PI", repr(math.pi)).replace("Math.E", repr(math.e))
    e = re.sub(r"Math\.(\w+)", r"math.\1", e)
    if not re.fullmatch(r"[-+*/().\deEmathpisqrtlog_ ]+", e):
        raise ValueError(f"unexpected numeric expression {expr!r}")
    return float(eval(e, {"__builtins__": {}, "math": math}))


def _strip_comments(s: str) -> str:
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def generate(ref_root: str) -> dict:
    src = os.path.join(ref_root, "src")
    vtxt = open(os.path.join(src, "variations.ts")).read()
    stxt = open(os.path.join(src, "serialize.ts")).read()
    ctxt = open(os.path.join(src, "variation-catalog-data.ts")).read()

    vblock = _strip_comments(_block(vtxt, "export const V = {"))
    index = {m.group(1): int(m.group(2)) for m in re.finditer(r"(\w+)\s*:\s*(\d+)\s*,", vblock)}
    names = {i: n for n, i in index.items()}
    assert sorted(names) == list(range(len(names))), "V indices must be dense"

    pblock = _strip_comments(_block(stxt, "export const VARIATION_PARAMS"))
    params = {}
    for m in re.finditer(r"(\w+)\s*:\s*\[([^\]]*)\]", pblock):
        params[m.group(1)] = re.findall(r"'([^']*)'", m.group(2))

    dblock = _strip_comments(_block(stxt, "export const VARIATION_DEFAULTS"))
    defaults = {}
    for m in re.finditer(r"(\w+)\s*:\s*\[([^\]]*)\]", dblock):
        defaults[m.group(1)] = [_num(x) for x in m.group(2).split(",") if x.strip()]

    dc_block = vtxt[vtxt.index("DC_VARIATION_SET"):]
    dc_block = _strip_comments(dc_block[: dc_block.index("]);")])
    dc = sorted(index[n] for n in re.findall(r"V\.(\w+)", dc_block))

    # ParamDoc ranges per catalog entry (entries start at `idx: V.<name>`).
    ranges = {}
    starts = [(m.start(), m.group(1)) for m in re.finditer(r"idx:\s*V\.(\w+)", ctxt)]
    for k, (pos, name) in enumerate(starts):
        end = starts[k + 1][0] if k + 1 < len(starts) else len(ctxt)
        body = _strip_comments(ctxt[pos:end])
        k0 = body.find("params:")
        if k0 < 0:
            continue
        k0 = body.index("[", k0)
        depth, k1 = 0, k0
        for k1 in range(k0, len(body)):
            depth += {"[": 1, "]": -1}.get(body[k1], 0)
            if depth == 0:
                break
        docs = []
        for d in re.finditer(r"\{([^{}]*)\}", body[k0 + 1:k1]):
            fields = dict(re.findall(r"(\w+)\s*:\s*('[^']*'|[^,]+)", d.group(1)))
            if "name" not in fields:
                continue
            docs.append({
                "name": fields["name"].strip("'"),
                "default": _num(fields.get("default", "0")),
                "min": _num(fields.get("min", "0")),
                "max": _num(fields.get("max", "0")),
            })
        ranges[name] = docs

    out = []
    for i in range(len(names)):
        n = names[i]
        pnames = params.get(n, [])
        docs = {d["name"]: d for d in ranges.get(n, [])}
        prange = []
        for p in pnames:
            d = docs.get(p)
            prange.append([d["min"], d["max"], d["default"]] if d else None)
        out.append({
            "idx": i,
            "name": n,
            "params": pnames,
            "defaults": defaults.get(n, [0.0] * len(pnames)),
            "ranges": prange,
            "dc": i in dc,
        })
    # Ken Perlin's improved-noise permutation as the reference's dc_perlin
    # uses it (src/shaders/noise_perlin.wgsl:12, 256 entries repeated).
    ptxt = open(os.path.join(src, "shaders", "noise_perlin.wgsl")).read()
    a = ptxt.index("array<u32, 512>(")
    perm = [int(x) for x in re.findall(r"(\d+)u", ptxt[a:ptxt.index(");", a)])]
    assert len(perm) == 512 and perm[:256] == perm[256:]
    return {"count": len(out), "variations": out, "perlin_perm": perm[:256]}


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYR3_REFERENCE")
    if not root:
        sys.exit("usage: python -m pyr3_b200.catalog_gen REFERENCE_ROOT (or set PYR3_REFERENCE)")
    cat = generate(root)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "catalog.json")
    with open(path, "w") as f:
        json.dump(cat, f, indent=0, separators=(",", ":"))
        f.write("\n")
    print(f"wrote {cat['count']} variations to {path}")
