"""The build's list of chaos-module structures (pyr3_b200/precompile_shapes.json).

build() NVRTC-compiles, without a GPU, the chaos modules the GPU tests load,
so a GPU run starts without compiling; it reads their structures from that
JSON file and never imports the tests.  These CPU tests keep the list
complete: every genome structure the GPU tests render is in it, and a
structure's placeholder records generate the same kernel source as the real
genome.  Regenerate the list after adding a test genome:

    python tests/test_precompile_shapes.py
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

from pyr3_b200 import _lib, build as B, genome as G, workloads  # noqa: E402


def gpu_test_genomes():
    """Genomes whose modules the GPU tests load, beyond the product
    workloads that build() compiles anyway."""
    import test_gpu_parity as T

    lin = [G.Genome(xforms=[G.Xform(variations=[G.Variation(0, 1.0)]) for _ in range(n)],
                    palette=[(0, 0, 0, 0), (1, 1, 1, 1)]) for n in (1, 3, 12, 20, 128)]
    return lin + [T._wide_genome(), T._linear_genome(), T._linear_genome(n=5, seed=11, blowup=True),
                  T._exact_genome()] + workloads.batch_256()[:8]


def _source(g) -> str:
    gg = G.expand_for_gpu(g)
    xf = np.ascontiguousarray(G.pack_xforms(gg), np.float32)
    gc = _lib.GenomeC(_lib.ptr(xf), len(gg.xforms), G.final_slot(gg), None, 100.0, 0.0, 0.0, 0.0, 0, 0.0)
    return _source_c(gc)


def _source_c(gc) -> str:
    n = C.c_uint64()
    _lib.check(_lib.lib().pyr3_jit_source(C.byref(gc), None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    _lib.check(_lib.lib().pyr3_jit_source(C.byref(gc), buf, n.value + 1, C.byref(n)))
    return buf.value.decode()


def test_placeholder_records_generate_the_genome_source():
    for g in [workloads.headline_1080p(), workloads.motion_4k()[0], workloads.batch_256()[3]]:
        sh = B.genome_shape(g)
        buf = B._packed_from_shape(sh)
        nx = len(sh["xforms"])
        gc = _lib.GenomeC(_lib.ptr(buf), nx, nx if sh["final"] is not None else -1, None,
                          100.0, 0.0, 0.0, 0.0, 0, 0.0)
        assert _source_c(gc) == _source(g)


def test_precompile_list_covers_the_gpu_test_genomes():
    listed = {json.dumps(s, sort_keys=True) for s in json.load(open(B.SHAPES))["shapes"]}
    missing = [g.name for g in gpu_test_genomes() if json.dumps(B.genome_shape(g), sort_keys=True) not in listed]
    assert not missing, f"run python tests/test_precompile_shapes.py to add {missing}"


if __name__ == "__main__":
    shapes, seen = [], set()
    for g in gpu_test_genomes():
        s = B.genome_shape(g)
        k = json.dumps(s, sort_keys=True)
        if k not in seen:
            seen.add(k)
            shapes.append(s)
    with open(B.SHAPES, "w") as f:
        json.dump({"shapes": shapes}, f, separators=(",", ":"))
        f.write("\n")
    print(f"{len(shapes)} structures -> {B.SHAPES}")
