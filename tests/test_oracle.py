"""CPU: pin the oracle against the reference's golden vectors and its own
shader math, and check its host algorithms against the reference's tests.

Sources of truth
* tests/golden/isaac_golden.json   (reference tests/fixtures/isaac/golden.json)
* tests/golden/variations_flam3.json (reference tests/fixtures/variations/*.json,
  flam3-instrumented f64 outputs, tolerance table of src/variations.test.ts)
* the reference's WGSL compiled for the CPU (oracle/_ref, built from the
  reference checkout by oracle/build.py), when present.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _state(d):
    return O.isaac_state(d["randcnt"], d["randa"], d["randb"], d["randc"], d["randmem"], d["randrsl"])


@pytest.mark.parametrize("case", ["zero_seed", "ascending_seed", "mixed_seed"])
def test_isaac_golden(case):
    """src/isaac.test.ts:48-186: irandinit and one round, byte for byte."""
    g = json.load(open(os.path.join(GOLD, "isaac_golden.json")))[case]
    st = _state(g["seed"])
    O.lib().or_irandinit(st, 1)
    assert (st == _state(g["after_irandinit"])).all()
    O.lib().or_isaac_round(st)
    assert (st == _state(g["after_one_round"])).all()


def test_rand_formulas():
    """chaos-rng.gpu.test.ts:47-56: rand01 = (u & 0x0fffffff) / 268435455,
    rand_11 = ((u & 0x0fffffff) - 0x07ffffff) / 134217727 (f32)."""
    st = O.pack_isaac_states(1, 7)
    probe = st.copy()
    for _ in range(40):
        u = O.lib().or_isaac_irand(probe)
        v = O.lib().or_rand01(st)
        assert v == np.float32(np.float32(u & 0x0FFFFFFF) * np.float32(1.0 / 268435455.0))


def test_pack_isaac_states_walker_hash():
    """src/isaac.ts:194-229: walker w's stream is PCG32(seed ^ (w*2654435761+1))
    where the product is a JS double (exact below 2^53 / 2654435761)."""
    a = O.pack_isaac_states(4, 12345, base=0)
    b = np.concatenate([O.pack_isaac_states(1, 12345, base=w) for w in range(4)])
    assert (a == b).all()
    assert a[0] == 16  # randcnt after irandinit
    assert len({tuple(a[k * 36:(k + 1) * 36]) for k in range(4)}) == 4


def test_pick_table_splits():
    """src/chaos-xform-pick.test.ts:39-110."""
    G = O.GRAIN
    half = G // 2
    rows = O.pack_xform_distrib([1.0, 1.0])
    row0, fb = rows[:G], rows[2 * G:]
    assert row0[0] == 0 and row0[half - 1] == 0 and row0[half] == 1 and row0[G - 1] == 1
    assert fb[half - 1] == 0 and fb[half] == 1
    rows = O.pack_xform_distrib([3.0, 1.0])
    c0 = int((rows[:G] == 0).sum())
    assert abs(c0 - 0.75 * G) <= 1 and int((rows[:G] == 1).sum()) + c0 == G
    rows = O.pack_xform_distrib([1.0, 1.0], xaos=[[1, 0], [1, 1]])
    assert (rows[:G] == 0).all()
    assert rows[G + half - 1] == 0 and rows[G + half] == 1
    with pytest.raises(ValueError):
        O.pack_xform_distrib([1.0, -1.0])


def test_calibration():
    """src/calibration.test.ts:5-56."""
    k1, k2 = O.derive_calibration(200, 16e6, 20)
    assert k1 == pytest.approx(20 * 255 * 268 / 256, rel=1e-12)
    assert k2 == pytest.approx(200 * 200 / (255 * 16e6), rel=1e-12)
    _, a = O.derive_calibration(200, 16e6, 1, 1)
    _, b = O.derive_calibration(200, 16e6, 1, 4)
    assert b / a == pytest.approx(16, rel=1e-12)


def test_kernel_norm_weights_sum_to_one():
    """src/density.test.ts:37-81: each radius' normalised kernel sums to 1."""
    lut = O.kernel_norm_lut()
    for r in (1, 2, 5, 11, 31, 64):
        s = sum(np.exp(-(dx * dx + dy * dy) / (2 * (r / 3) ** 2))
                for dy in range(-r, r + 1) for dx in range(-r, r + 1) if dx * dx + dy * dy <= r * r)
        assert s / lut[r] == pytest.approx(1.0, rel=1e-6)
    assert lut[0] == 1.0


def test_spatial_kernel():
    """src/spatial-filter.test.ts: parity rule and normalisation."""
    for os_, fw in ((1, 3), (2, 4), (3, 5), (4, 8)):
        k = O.spatial_kernel(0.5, os_)
        assert len(k) == fw and ((len(k) ^ os_) & 1) == 0
        assert float(k.sum()) == pytest.approx(1.0, abs=1e-6)
        assert np.allclose(k, k[::-1])


def test_compute_dispatch():
    """src/renderer.ts:57-78 for the configurations' sizes."""
    assert O.compute_dispatch(50, 640, 480) == (1024, 15000, 15360000)
    assert O.compute_dispatch(500, 1920, 1080) == (1024, 1012500, 1036800000)
    w, it, s = O.compute_dispatch(2000, 3840, 2160)
    assert it == 1048576 and s >= 2000 * 3840 * 2160
    assert O.compute_dispatch(1, 64, 64) == (1, 4096, 4096)
    assert O.compute_dispatch(4, 64, 64, walkers_override=7) == (7, 2341, 16387)


def test_splat_saturates():
    """src/chaos-saturate.gpu.test.ts: counts pin at 2^32-1, never wrap."""
    pal = np.ones(1024, np.float32)
    hist = np.zeros(4 * 4 * 4, np.uint32)
    hist[:] = 0xFFFFFF00
    pts = np.array([[0.0, 0.0, 0.5, 1.0]] * 3, np.float32)
    O.splat_points(pts, 4, 4, 1.0, 0.0, 0.0, 0.0, 0, pal, hist)
    cell = hist.reshape(4, 4, 4)[2, 2]
    assert (cell == 0xFFFFFFFF).all()


@pytest.mark.skipif(not O.ref_available(), reason="reference shaders not compiled here")
def test_reference_variations_match_flam3_goldens():
    """The reference's WGSL variations (compiled for the CPU) reproduce the
    flam3 f64 fixtures within f32 accuracy; RNG-branch fixtures pass when any
    seeded branch matches (src/variations.test.ts runMultiBranchRng)."""
    fx = json.load(open(os.path.join(GOLD, "variations_flam3.json")))
    # popcorn2: sin(tan(c*y)) is ill-conditioned near the tan poles in f32.
    loose = {"popcorn2": 2e-3}
    bad = []
    for f in fx:
        if f["runner"] == "smoke":
            continue
        af = f["affine"]
        a0 = np.array([af.get("a", 1), af.get("b", 0), af.get("c", 0), 1], np.float32)
        a1 = np.array([af.get("d", 0), af.get("e", 1), af.get("f", 0), 1], np.float32)
        p = np.array(f["params"], np.float32)
        tol = loose.get(f["name"], 1e-4)
        tries = 48 if f["runner"] in ("branch", "julia") else 1
        for tx, ty, w, ex, ey in f["rows"]:
            ok = False
            for t in range(tries):
                out = O.ref_eval_grid(f["idx"], [tx, ty], w, p, a0, a1, O.pack_isaac_states(1, 99 + t))[0]
                err = max(abs(out[0] - ex), abs(out[1] - ey)) / max(1.0, abs(ex), abs(ey))
                if err <= tol:
                    ok = True
                    break
            if not ok:
                bad.append((f["name"], tx, ty))
    assert not bad, bad[:10]


@pytest.mark.skipif(not O.ref_available(), reason="reference shaders not compiled here")
def test_density_and_visualize_restatement_match_reference():
    """oracle.c's density / visualize equal the reference's WGSL on the CPU."""
    rng = np.random.default_rng(5)
    W, H = 48, 40
    hist = np.zeros((H, W, 4), np.uint32)
    cnt = rng.integers(0, 6, (H, W)) * 255
    cnt[rng.random((H, W)) < 0.4] = 0
    hist[..., 3] = cnt
    for ch in range(3):
        hist[..., ch] = (cnt * rng.random((H, W))).astype(np.uint32)
    hist = hist.reshape(-1)
    k1, k2 = O.derive_calibration(40, 5e4, 4)
    a = O.density(hist, W, H, 9 * 1 + 1, 0 * 1 + 1, 0.4, k1, k2)
    b = O.ref_density(hist, W, H, 10.0, 1.0, 0.4, k1, k2)
    assert np.array_equal(a, b)
    kern = O.spatial_kernel(0.5, 2)
    args = (W // 2, H // 2, 2, kern, k1, k2, 4.0, 1.0, 1.0, 0.01)
    v1 = O.visualize(*args, src_u32=hist)
    v2 = O.ref_visualize(*args, src_u32=hist)
    assert np.array_equal(v1, v2)
    v1 = O.visualize(*args, src_f32=a)
    v2 = O.ref_visualize(*args, src_f32=a)
    assert np.array_equal(v1, v2)


def _curves_and_hsl():
    from pyr3_b200 import genome as G

    curves = {"composite": [(0, 0.05), (0.5, 0.6), (1, 1)], "r": [(0, 0), (1, 0.9)],
              "g": [(0, 0), (1, 1)], "b": [(0, 0.1), (0.3, 0.2), (0.7, 0.8), (1, 1)],
              "luma": [(0, 0), (0.4, 0.5), (1, 1)]}
    return G.bake_curves(curves), G.curves_active_mask(curves), (37.0, 1.3, -0.05)


@pytest.mark.skipif(not O.ref_available(), reason="reference shaders not compiled here")
def test_visualize_curves_and_hsl_restatement_matches_reference():
    """oracle.c's colour curves + HSL adjustment (visualize_u32.wgsl:217-243)
    equal the reference's WGSL on the CPU, for u32 and f32 sources."""
    rng = np.random.default_rng(6)
    W, H = 48, 40
    hist = np.zeros((H, W, 4), np.uint32)
    cnt = rng.integers(0, 9, (H, W)) * 255
    cnt[rng.random((H, W)) < 0.3] = 0
    hist[..., 3] = cnt
    for ch in range(3):
        hist[..., ch] = (cnt * rng.random((H, W))).astype(np.uint32)
    hist = hist.reshape(-1)
    k1, k2 = O.derive_calibration(40, 5e4, 4)
    lut, mask, hsl = _curves_and_hsl()
    assert mask == 0b11011
    kern = O.spatial_kernel(0.5, 2)
    args = (W // 2, H // 2, 2, kern, k1, k2, 4.0, 1.0, 1.0, 0.01)
    for kw in ({"curves_active": mask, "curves": lut}, {"hsl": hsl},
               {"curves_active": mask, "curves": lut, "hsl": hsl}):
        v1 = O.visualize(*args, src_u32=hist, **kw)
        v2 = O.ref_visualize(*args, src_u32=hist, **kw)
        assert np.array_equal(v1, v2), kw
        assert not np.array_equal(v1, O.visualize(*args, src_u32=hist))
    a = O.density(hist, W, H, 10.0, 1.0, 0.4, k1, k2)
    kw = {"curves_active": mask, "curves": lut, "hsl": hsl}
    assert np.array_equal(O.visualize(*args, src_f32=a, **kw), O.ref_visualize(*args, src_f32=a, **kw))


def test_bake_curves_matches_reference_cases():
    """src/channel-curves.test.ts: activeMask bits, identity / inverse
    bakes, end clamps."""
    from pyr3_b200 import genome as G

    ident = [(0, 0), (1, 1)]
    lift = [(0, 0.1), (1, 1)]
    assert G.curves_active_mask(None) == 0
    names = G.CURVE_CHANNELS
    assert G.curves_active_mask({n: ident for n in names}) == 0
    for i, n in enumerate(names):
        assert G.curves_active_mask({m: (lift if m == n else ident) for m in names}) == 1 << i
    assert G.curves_active_mask({n: lift for n in names}) == 0b11111
    one = {n: ident for n in names}
    one["composite"] = [(0, 1), (1, 0)]
    lut = G.bake_curves(one)
    assert np.allclose(lut[:256], 1 - np.arange(256) / 255, atol=5e-3)
    assert np.allclose(lut[256:512], np.arange(256) / 255, atol=5e-3)
    one["composite"] = [(0.25, 0.5), (1, 1)]
    lut = G.bake_curves(one)
    assert lut[0] == pytest.approx(0.5, abs=1e-3) and lut[63] == pytest.approx(0.5, abs=1e-3)
    one["composite"] = [(0, 0), (0.75, 0.5)]
    assert G.bake_curves(one)[200] == pytest.approx(0.5, abs=1e-3)


from refrender import TONEMAP_CASES  # noqa: E402


@pytest.mark.skipif(not O.ref_available(), reason="reference shaders not compiled here")
@pytest.mark.parametrize("tm", TONEMAP_CASES, ids=lambda t: f"g{t[0]}-v{t[1]}-hp{t[2]}-bg{sum(t[3]) > 0:d}-tr{t[4]:d}")
def test_visualize_parameter_space_restatement_matches_reference(tm):
    """oracle.c's visualize equals the reference's WGSL on the CPU across
    gamma, vibrancy, highlight power, background and transparency, for u32
    (density estimation off) and f32 (density-estimated) sources at
    oversample 1 and 2."""
    gamma, vib, hp, bg, transparent = tm
    rng = np.random.default_rng(7)
    for os_ in (1, 2):
        W, H = 24 * os_, 20 * os_
        hist = np.zeros((H, W, 4), np.uint32)
        cnt = rng.integers(0, 40, (H, W)) * 255
        cnt[rng.random((H, W)) < 0.3] = 0
        hist[..., 3] = cnt
        for ch in range(3):
            hist[..., ch] = (cnt * rng.random((H, W))).astype(np.uint32)
        hist = hist.reshape(-1)
        k1, k2 = O.derive_calibration(40, 5e4, 4, os_)
        args = (W // os_, H // os_, os_, O.spatial_kernel(0.5, os_), k1, k2, gamma, vib, hp, 0.01)
        kw = {"bg": bg, "transparent": transparent}
        v1 = O.visualize(*args, src_u32=hist, **kw)
        assert np.array_equal(v1, O.ref_visualize(*args, src_u32=hist, **kw))
        a = O.density(hist, W, H, 9.0 * os_ + 1, 1.0, 0.4, k1, k2)
        assert np.array_equal(O.visualize(*args, src_f32=a, **kw), O.ref_visualize(*args, src_f32=a, **kw))


@pytest.mark.skipif(not O.ref_available(), reason="reference shaders not compiled here")
def test_draw_free_variations_draw_nothing_in_the_reference():
    """The build marks which variations may draw from the walker's stream
    (pyr3_b200.build.rng_variations, used to skip a draw-free final xform
    during the burn-in).  Every variation the library marks draw-free
    leaves the ISAAC state unchanged in the reference's apply_variation
    (chaos.wgsl:7731) on a seeded grid with random parameters."""
    from pyr3_b200 import build as B, genome as G

    draws = B.rng_variations()
    cat = G.catalog()
    wrong = []
    for v in cat:
        if v["name"] in draws or v["dc"] or v["idx"] == 97:
            continue
        rng = np.random.default_rng(v["idx"])
        pts = rng.uniform(-2.0, 2.0, (256, 2)).astype(np.float32)
        p = np.zeros(10, np.float32)
        for k, rg in enumerate(v["ranges"][:10]):
            if rg:
                p[k] = rng.uniform(rg[0], rg[1]) if rg[1] > rg[0] else rg[0]
        a0 = np.array([0.8, -0.4, 0.1, 1.0], np.float32)
        a1 = np.array([0.3, 0.5, 0.2, 1.0], np.float32)
        st = O.pack_isaac_states(256, 3 + v["idx"])
        st2 = st.copy()
        O.ref_eval_grid(v["idx"], pts, 0.75, p, a0, a1, st2)
        if not np.array_equal(st, st2):
            wrong.append(v["name"])
    assert not wrong, wrong
    assert 60 <= len(draws) <= 90
