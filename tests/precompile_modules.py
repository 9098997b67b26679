"""Build step: NVRTC-compile, without a GPU, the chaos modules and variation
evaluators that the GPU tests, smoke() and the benches load, into the
package's cubin cache (pyr3_b200/_cubins, which the library prefers when it
exists), so a GPU run starts without compiling.

    python tests/precompile_modules.py
"""
import ctypes as C
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)


def genomes():
    from pyr3_b200 import genome as G, workloads
    import test_gpu_parity as T

    lin = [G.Genome(xforms=[G.Xform(variations=[G.Variation(0, 1.0)]) for _ in range(n)],
                    palette=[(0, 0, 0, 0), (1, 1, 1, 1)]) for n in (1, 3, 12, 20, 128)]
    return lin + [workloads.plain_small(), workloads.headline_1080p(), workloads.motion_4k()[0],
                  T._wide_genome(), T._linear_genome(), T._linear_genome(n=5, seed=11, blowup=True)] + \
        workloads.denoise_set(seed=5, n=72, size=256)[:4]


def precompile(verbose: bool = True) -> None:
    from pyr3_b200 import _lib, renderer as R

    L = _lib.lib()
    t = time.time()
    bad = 0
    for i in range(326):
        impl, dc, nm = C.c_int32(), C.c_int32(), C.c_char_p()
        L.pyr3_variation_info(i, C.byref(impl), C.byref(dc), C.byref(nm))
        if impl.value and L.pyr3_jit_compile_variation(i, C.byref(C.c_uint64())) != 0:
            bad += 1
    for g in genomes():
        gg = R.GpuGenome(g)
        for agg in (0, 1):
            if L.pyr3_jit_compile(C.byref(gg.c), agg, C.byref(C.c_uint64())) != 0:
                bad += 1
    if bad:
        raise RuntimeError(f"{bad} modules failed to compile: {L.pyr3_last_error().decode()[:400]}")
    if verbose:
        print(f"precompiled modules in {time.time() - t:.0f} s")


if __name__ == "__main__":
    precompile()
