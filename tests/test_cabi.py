"""CPU: the C-ABI library loads, exports every function include/pyr3.h
declares, its host-side math matches the oracle, and the NVRTC-specialised
chaos kernel / variation evaluators compile for sm_100a (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from pyr3_b200 import _lib, genome as G, renderer as R, workloads

HDR = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "pyr3.h")


def test_library_exports_every_header_symbol():
    names = set(re.findall(r"^\s*(?:int|uint64_t|const char \*)\s*\*?\s*(pyr3_\w+)\s*\(", open(HDR).read(), re.M))
    assert len(names) >= 25
    L = _lib.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing
    assert names == set(_lib.exported_symbols())


def test_pick_table_matches_oracle():
    rng = np.random.default_rng(1)
    for n in (1, 2, 3, 12, 40, 128):
        w = rng.uniform(0.0, 1.0, n).astype(np.float32)
        w[rng.random(n) < 0.1] = 0.0
        xa = None
        if n > 1 and n % 2 == 0:
            xa = rng.uniform(0.0, 2.0, (n, n)).astype(np.float32)
            xa[rng.random((n, n)) < 0.2] = 0.0
        out = np.zeros((n + 1) * O.GRAIN, np.uint32)
        _lib.check(_lib.lib().pyr3_pick_table(n, _lib.ptr(w), _lib.ptr(xa) if xa is not None else None,
                                              _lib.ptr(out)))
        ref = O.pack_xform_distrib(w.astype(np.float64), None if xa is None else xa.astype(np.float64))
        assert np.array_equal(out, ref), n


def test_bake_lut_and_dispatch_match_oracle():
    rng = np.random.default_rng(2)
    stops = sorted([(0.0, *rng.random(3))] + [(float(t), *rng.random(3)) for t in rng.random(5)] +
                   [(1.0, *rng.random(3))])
    for mode, k in (("linear", 0), ("step", 1), ("smooth", 2)):
        assert np.array_equal(G.bake_lut(stops, 0.0, mode), O.bake_lut(stops, k))
    for spp, w, h in ((50, 640, 480), (500, 1920, 1080), (2000, 3840, 2160), (3, 32, 32)):
        assert R.compute_dispatch(spp, w, h) == O.compute_dispatch(spp, w, h)


def test_pack_xforms_layout():
    """src/genome.ts:293-421 record layout."""
    g = workloads.headline_1080p()
    buf = G.pack_xforms(g).reshape(-1, 116)
    assert buf.shape[0] == 13
    x = g.xforms[3]
    rec = buf[3]
    assert np.allclose(rec[[0, 1, 2, 3, 4, 5, 6]], np.float32([x.a, x.b, x.c, x.weight, x.d, x.e, x.f]))
    assert rec[7] == len(x.variations) and rec[15] == 1.0
    for k, v in enumerate(x.variations):
        assert rec[20 + 4 * k] == v.index
        assert rec[22 + 4 * k] == np.float32(v.params[0])
        assert rec[52 + 4 * k] == np.float32(v.params[2])
        assert rec[84 + 4 * k + 3] == np.float32(v.params[9])
    assert G.final_slot(g) == 12


def test_symmetry_expansion():
    g = workloads.plain_small()
    g.symmetry = ("dihedral", 4)
    e = G.expand_for_gpu(g)
    assert len(e.xforms) == 3 + 1 + 3 and e.symmetry is None
    assert (e.xforms[3].a, e.xforms[3].e) == (-1.0, 1.0)
    assert e.xforms[4].a == 0.0 and e.xforms[4].b == -1.0  # 90 degree rotation, round6
    assert g.symmetry == ("dihedral", 4)  # input untouched


def test_json_roundtrip():
    g = workloads.headline_1080p()
    j = G.genome_to_json(g)
    g2 = G.genome_from_json(j)
    assert np.array_equal(G.pack_xforms(g), G.pack_xforms(g2))


def test_jit_compiles_plain_small():
    gg = R.GpuGenome(workloads.plain_small())
    n = C.c_uint64()
    _lib.check(_lib.lib().pyr3_jit_compile(C.byref(gg.c), 0, C.byref(n)))
    assert n.value > 10000
    _lib.check(_lib.lib().pyr3_jit_compile(C.byref(gg.c), 1, C.byref(n)))  # aggregated scatter


def test_jit_rejects_malformed_genome():
    g = workloads.plain_small()
    gg = R.GpuGenome(g)
    bad = _lib.GenomeC(gg.c.xforms, 0, -1, None, 1.0, 0.0, 0.0, 0.0, 0, 0.0)
    n = C.c_uint64()
    assert _lib.lib().pyr3_jit_compile(C.byref(bad), 0, C.byref(n)) == _lib.PYR3_E_INVALID
    xf = gg.xforms.copy()
    xf[7] = np.nan
    gbad = _lib.GenomeC(_lib.ptr(xf), 3, -1, None, 1.0, 0.0, 0.0, 0.0, 0, 0.0)
    assert _lib.lib().pyr3_jit_compile(C.byref(gbad), 0, C.byref(n)) == _lib.PYR3_E_INVALID
    assert b"variation count" in _lib.lib().pyr3_last_error()


def _implemented():
    out = []
    for i in range(326):
        impl, dc = C.c_int32(), C.c_int32()
        nm = C.c_char_p()
        _lib.check(_lib.lib().pyr3_variation_info(i, C.byref(impl), C.byref(dc), C.byref(nm)))
        if impl.value:
            out.append(i)
    return out


def test_variation_evaluators_compile():
    """A spread of the implemented variations NVRTC-compile (cached on disk)."""
    ids = _implemented()
    assert len(ids) >= 97
    for i in ids[:: max(1, len(ids) // 12)]:
        n = C.c_uint64()
        rc = _lib.lib().pyr3_jit_compile_variation(i, C.byref(n))
        assert rc == 0, _lib.lib().pyr3_last_error()


def test_committed_genome_files_match_the_generator(tmp_path):
    """pyr3_b200/genomes/*.pyr3.json (the benchmark genomes in the
    reference's file format, so the reference can render them) are what
    the seeded generator writes today."""
    import os

    from pyr3_b200 import workloads

    here = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pyr3_b200", "genomes")
    fresh = workloads.write_all(str(tmp_path))
    assert sorted(os.listdir(here)) == sorted(os.path.basename(p) for p in fresh)
    for p in fresh:
        assert open(p).read() == open(os.path.join(here, os.path.basename(p))).read(), p
