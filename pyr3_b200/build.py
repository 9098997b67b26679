"""Build libpyr3cuda.so in-tree (sm_100a).

1. Embed the NVRTC sources (csrc/jit/*.cuh) and the variation table
   (catalog.json names; which variations / direct colours the library
   implements, found by scanning the VAR(...) / DCV(...) definitions) into
   csrc/gen/jit_sources.inc.
2. nvcc -gencode arch=compute_100a,code=sm_100a the C-ABI (capi.cpp), the
   JIT driver (jit.cpp), the density / tonemap passes (passes.cu), the
   fixed scratch of the allocation-free present (noalloc.cu) and the
   denoiser layers (denoise.cu).
"""
from __future__ import annotations

import glob
import json
import os
import re
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
JIT = os.path.join(CSRC, "jit")
GEN = os.path.join(CSRC, "gen")
LIB = os.path.join(PKG, "libpyr3cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = "/usr/local/cuda/lib64"


def _strip(src: str) -> str:
    return "\n".join(l for l in src.splitlines() if l.strip() != "#pragma once")


def _raw(s: str) -> str:
    # Raw string literals, split so no single literal gets unwieldy.
    parts = []
    chunk = 60000
    for i in range(0, len(s), chunk):
        parts.append('R"PYR3SRC(' + s[i:i + chunk] + ')PYR3SRC"')
    return "\n".join(parts) if parts else '""'


_DRAWS = re.compile(r"\b(RAND01|RAND11|IRAND|rand01|rand_11|irand)\s*\(|[(,]\s*c\s*[),]")


def rng_variations(vsrc=None) -> set:
    """Names of the library's variations that may draw from the walker's
    random stream: every VAR body that uses an RNG macro or passes the
    context (which holds the stream) to another function.  The rest draw
    nothing, whatever their parameters."""
    if vsrc is None:
        vsrc = [open(f).read() for f in sorted(glob.glob(os.path.join(JIT, "vlib_*.cuh")))
                if not f.endswith("vlib_core.cuh")]
    parts = re.split(r"^(VAR|DCV)\((\w+)\)", "\n".join(vsrc), flags=re.M)
    return {parts[i + 1] for i in range(1, len(parts), 3) if parts[i] == "VAR" and _DRAWS.search(parts[i + 2])}


def generate_sources() -> str:
    os.makedirs(GEN, exist_ok=True)
    core = _strip(open(os.path.join(JIT, "vlib_core.cuh")).read())
    vlibs = sorted(f for f in glob.glob(os.path.join(JIT, "vlib_*.cuh")) if not f.endswith("vlib_core.cuh"))
    vsrc = [_strip(open(f).read()) for f in vlibs]
    chaos = _strip(open(os.path.join(JIT, "chaos_kernel.cuh")).read())
    marker = "// ==== PYR3 KERNEL SECTION ===="
    pre, kern = chaos.split(marker, 1)
    ev = _strip(open(os.path.join(JIT, "eval_kernel.cuh")).read())
    cat = json.load(open(os.path.join(PKG, "catalog.json")))["variations"]
    names = [v["name"] for v in cat]
    allsrc = "\n".join(vsrc)
    impl = set(re.findall(r"^VAR\((\w+)\)", allsrc, re.M))
    dcs = set(re.findall(r"^DCV\((\w+)\)", allsrc, re.M))
    unknown = (impl | dcs) - set(names)
    if unknown:
        raise RuntimeError(f"variation library defines names not in the catalog: {sorted(unknown)}")
    perm = json.load(open(os.path.join(PKG, "catalog.json")))["perlin_perm"]
    core += ("\n__device__ const unsigned char c_perlin_perm[256] = {" +
             ", ".join(str(v) for v in perm) + "};\n")
    out = ["// generated by pyr3_b200/build.py -- do not edit"]
    out.append(f"static const char* const kSrcCore = {_raw(core)};")
    out.append(f"static const int kNumVlib = {len(vsrc)};")
    out.append("static const char* const kSrcVlib[] = {" + ",\n".join(_raw(s) for s in vsrc) + "};")
    out.append(f"static const char* const kSrcChaosPre = {_raw(pre)};")
    out.append(f"static const char* const kSrcChaosKernel = {_raw(kern)};")
    out.append(f"static const char* const kSrcEval = {_raw(ev)};")
    out.append("static const char* const kVarNames[326] = {" + ", ".join(f'"{n}"' for n in names) + "};")
    out.append("static const unsigned char kVarImpl[326] = {" +
               ", ".join("1" if n in impl else "0" for n in names) + "};")
    out.append("static const unsigned char kVarDc[326] = {" +
               ", ".join("1" if n in dcs else "0" for n in names) + "};")
    draws = rng_variations(vsrc)
    out.append("static const unsigned char kVarRng[326] = {" +
               ", ".join("1" if n in draws else "0" for n in names) + "};")
    text = "\n".join(out) + "\n"
    path = os.path.join(GEN, "jit_sources.inc")
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as f:
            f.write(text)
    return path


def build(force: bool = False) -> str:
    inc = generate_sources()
    srcs = [os.path.join(CSRC, f) for f in ("capi.cpp", "jit.cpp", "passes.cu", "noalloc.cu", "denoise.cu")]
    deps = srcs + [inc, os.path.join(ROOT, "include", "pyr3.h"), os.path.join(CSRC, "jit.h"),
                   os.path.join(CSRC, "passes.h"), os.path.join(CSRC, "noalloc.h"),
                   os.path.join(CSRC, "denoise.h")]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    cmd = [NVCC, "-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, *srcs, "-o", LIB,
           "-cudart", "static", "-L", CUDA_LIB, "-lnvrtc", "-ldl", "-lpthread",
           "-Xlinker", f"-rpath,{CUDA_LIB}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return LIB


CUBINS = os.path.join(PKG, "_cubins")
SHAPES = os.path.join(PKG, "precompile_shapes.json")


def make_cubin_cache() -> str:
    """The in-package cubin cache the library uses when PYR3_CACHE_DIR is
    unset (filled by precompile())."""
    os.makedirs(CUBINS, exist_ok=True)
    return CUBINS


def genome_shape(g) -> dict:
    """The structure of a genome that selects its specialised chaos module:
    per xform the variation indices and whether it has a post affine, and
    the same for the final xform (None without one)."""
    from .genome import expand_for_gpu

    gg = expand_for_gpu(g)

    def one(x):
        return {"vars": [int(v.index) for v in x.variations[:8]], "post": x.post is not None}

    fin = gg.finalxform if (gg.finalxform is not None and gg.finalxform.active) else None
    return {"xforms": [one(x) for x in gg.xforms], "final": one(fin) if fin is not None else None}


def _packed_from_shape(shape):
    """Packed xform records (the reference's 116-float layout) of a
    structure, every numeric value a placeholder: enough to compile its
    module, since the generated code depends only on the structure."""
    import numpy as np

    xs = shape["xforms"] + ([shape["final"]] if shape["final"] is not None else [])
    buf = np.zeros(len(xs) * 116, np.float32)
    for i, x in enumerate(xs):
        o = i * 116
        buf[o + 0], buf[o + 3], buf[o + 4 + 3], buf[o + 10] = 1.0, 1.0, len(x["vars"]), 1.0
        buf[o + 5] = 1.0
        if x["post"]:
            buf[o + 12], buf[o + 15], buf[o + 17] = 1.0, 1.0, 1.0
        for k, v in enumerate(x["vars"]):
            buf[o + 20 + 4 * k], buf[o + 21 + 4 * k] = v, 1.0
    return buf


def product_genomes() -> list:
    """Genomes of the product's own workloads whose modules the smoke run
    and the benches load."""
    from . import workloads

    return [workloads.plain_small(), workloads.headline_1080p(), workloads.motion_4k()[0]] + \
        workloads.denoise_set(seed=5, n=72, size=256)[:4]


def precompile(verbose: bool = True, extra_shapes=None) -> int:
    """NVRTC-compile (no GPU needed) every variation evaluator and the chaos
    modules of the product workloads and of the structures listed in
    precompile_shapes.json (those the GPU tests render), both scatter
    variants each, into the cubin cache; returns the number of modules."""
    import ctypes as C
    import time

    from . import _lib
    from .renderer import GpuGenome

    L = _lib.lib()
    t = time.time()
    bad = n = 0
    for i in range(326):
        impl, dc, nm = C.c_int32(), C.c_int32(), C.c_char_p()
        L.pyr3_variation_info(i, C.byref(impl), C.byref(dc), C.byref(nm))
        if impl.value:
            n += 1
            if L.pyr3_jit_compile_variation(i, C.byref(C.c_uint64())) != 0:
                bad += 1
    shapes = [genome_shape(g) for g in product_genomes()]
    if os.path.exists(SHAPES):
        shapes += json.load(open(SHAPES))["shapes"]
    shapes += list(extra_shapes or [])
    seen = set()
    for sh in shapes:
        key = json.dumps(sh, sort_keys=True)
        if key in seen:
            continue
        seen.add(key)
        buf = _packed_from_shape(sh)
        nx = len(sh["xforms"])
        gc = _lib.GenomeC(_lib.ptr(buf), nx, nx if sh["final"] is not None else -1, None,
                          100.0, 0.0, 0.0, 0.0, 0, 0.0)
        for agg in (0, 1):
            n += 1
            if L.pyr3_jit_compile(C.byref(gc), agg, C.byref(C.c_uint64())) != 0:
                bad += 1
    if bad:
        raise RuntimeError(f"{bad} modules failed to compile: {L.pyr3_last_error().decode()[:400]}")
    if verbose:
        print(f"precompiled {n} modules in {time.time() - t:.0f} s")
    return n


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
