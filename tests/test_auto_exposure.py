"""Render-time auto-exposure (src/auto-exposure.ts, bin/pyr3-render.ts:
487-513).

CPU: the oracle against the reference's own unit-test cases
(src/auto-exposure.test.ts, src/presets.test.ts), and the library's fit
logic (pyr3_fit_brightness, host code) against the same cases and against
the oracle on random fits.  GPU: the device luminance sum against the oracle
and the exact integer mean, and the device re-present loop against the
oracle's loop driven by host presents."""
import copy
import ctypes as C
import math
from fractions import Fraction

import numpy as np
import pytest

from oracle import auto_exposure as OA
from pyr3_b200 import _lib, auto_exposure as AE, genome as G, renderer as R, workloads

FITS = [("oracle", lambda *a: OA.fit_brightness_to_target(*a)[0]),
        ("library", lambda *a: tuple(vars(AE.fit_brightness_to_target(*a)).values()))]


def _half(vals):
    return np.asarray(vals, np.float32).astype(np.float16)


# ---------------------------------------------------------------- CPU

def test_mean_luminance_reference_cases():
    """src/auto-exposure.test.ts:34-83."""
    assert OA.mean_luminance(np.zeros(0, np.uint8)) == 0
    assert OA.mean_luminance(np.array([0, 0, 0, 255, 0, 0, 0, 255], np.uint8)) == 0
    assert OA.mean_luminance(np.array([255, 255, 255, 255], np.uint8)) == 255
    assert OA.mean_luminance(np.array([60, 90, 120, 255, 0, 0, 0, 255], np.uint8)) == 45
    assert OA.mean_luminance_half(np.zeros(0, np.float16)) == 0
    assert OA.mean_luminance_half(_half([1, 1, 1, 1])) == pytest.approx(255, abs=5e-5)
    assert OA.mean_luminance_half(_half([4, 4, 4, 1])) == pytest.approx(255, abs=5e-5)
    assert OA.mean_luminance_half(_half([0.5, 0.5, 0.5, 1])) == pytest.approx(127.5, abs=0.05)
    nan = np.array([0x7E00, 0x7E00, 0x7E00, 0], np.uint16).view(np.float16)
    assert OA.mean_luminance_half(nan) == 0
    # rgba32f read as rgba16float: 65519 rounds to 65504 (finite, clamps to
    # 1); 65520 rounds to +inf, which the clamp maps to 0.
    assert OA.mean_luminance_rgba32f(np.array([65519, 65520, -3, 0], np.float32)) == pytest.approx(85.0)


@pytest.mark.parametrize("name,fit", FITS, ids=[f[0] for f in FITS])
def test_fit_reference_cases(name, fit):
    """src/auto-exposure.test.ts:85-157, against the oracle and the library."""
    calls = []

    def never(b):
        calls.append(b)
        return 0.0

    r = fit(3.0, 100.0, 100 * (1 + OA.AE_DEADBAND / 2), never)
    assert r[:3] == (3.0, False, 0) and calls == []
    assert fit(3.0, 100.0, 0.0, lambda b: 100.0)[:2] == (3.0, False)
    assert fit(3.0, 0.0, 50.0, lambda b: 100.0)[1] is False
    for t, i in ((math.nan, 50.0), (100.0, math.nan)):
        r = fit(3.0, t, i, never)
        assert r[:2] == (3.0, False) and calls == []
    r = fit(1.0, 80.0, 10.0, lambda b: b * 10)
    assert r[1] is True and r[0] == pytest.approx(8.0, abs=1e-6) and r[3] == pytest.approx(80, abs=1e-6)
    assert r[2] == 1
    r = fit(1.0, 60.0, 30 * math.log(2), lambda b: 30 * math.log1p(b))
    assert r[1] is True and r[2] <= OA.AE_MAX_ITERS
    assert 1 - OA.AE_DEADBAND < r[3] / 60.0 < 1 + OA.AE_DEADBAND
    r = fit(1.0, 100.0, 5 * (1 - math.exp(-1 / 1e6)), lambda b: 5 * (1 - math.exp(-b / 1e6)))
    assert r[0] <= OA.AE_BRIGHTNESS_MAX and r[2] <= OA.AE_MAX_ITERS


def test_library_fit_matches_oracle_on_random_fits():
    """The same brightness sequence, bit for bit, over random bases, targets
    and response curves, including the NaN and non-positive responses the
    guards handle."""
    rng = np.random.default_rng(11)
    models = [lambda b, a: a * b, lambda b, a: a * math.log1p(b), lambda b, a: a * (1 - math.exp(-b)),
              lambda b, a: a * math.sqrt(b), lambda b, a: -1.0 if b > a else b,
              lambda b, a: math.nan if b > 2 * a else b * a]
    for k in range(300):
        base = float(rng.uniform(0.01, 10))
        a = float(rng.uniform(0.1, 50))
        model = models[k % len(models)]
        target = float(rng.uniform(0.5, 250))
        initial = model(base, a)
        seq_lib = []

        def rr(b, s=seq_lib, m=model, a=a):
            s.append(b)
            return m(b, a)

        ref, seq_ref = OA.fit_brightness_to_target(base, target, initial, lambda b, m=model, a=a: m(b, a))
        got = AE.fit_brightness_to_target(base, target, initial, rr)
        assert seq_lib == seq_ref
        exp = (got.brightness, got.corrected, got.iters, got.final_mean, got.factor)
        assert all((x == y) or (isinstance(x, float) and math.isnan(x) and math.isnan(y))
                   for x, y in zip(exp, ref)), (k, exp, ref)


def test_library_fit_raises_the_rerender_error():
    def boom(b):
        raise RuntimeError("present failed")

    with pytest.raises(RuntimeError, match="present failed"):
        AE.fit_brightness_to_target(1.0, 80.0, 10.0, boom)


def test_probe_preset_reference_cases():
    """applyPreset in force mode (src/presets.test.ts:78-121, the 4K spec,
    which is customSpec(3840, 200)) and the probe geometry of the oracle."""
    g = G.Genome(scale=220, quality=500, oversample=4, size=(800, 592))
    out = AE.apply_probe_preset(g, 3840, 200)
    assert out.size == (3840, 2841) and out.scale == pytest.approx(220 * 4.8, abs=1e-3)
    assert out.oversample == 1 and out.quality == 200
    out = AE.apply_probe_preset(G.Genome(scale=355.352, size=(1280, 720), quality=100), 3840, 200)
    assert out.size == (3840, 2160) and out.scale == pytest.approx(355.352 * 3, abs=1e-3)
    assert out.quality == 100
    out = AE.apply_probe_preset(G.Genome(size=None, quality=None, oversample=4), 3840, 200)
    assert out.size is None and out.oversample == 1 and out.quality == 200
    for size in ((640, 480), (480, 640), (1024, 1024), (300, 7), (2000, 999), None):
        g = G.Genome(scale=123.0, size=size, quality=50,
                     density={"maxRad": 9.0, "minRad": 1.0, "curve": 0.4})
        p = AE.apply_probe_preset(g)
        w, h, sc, de, q = OA.probe_geometry(size, 123.0, (9.0, 1.0), 50)
        assert (p.size or (1024, 1024)) == (w, h) and p.scale == sc and p.quality == q
        assert (p.density["maxRad"], p.density["minRad"]) == de


# ---------------------------------------------------------------- GPU

def _exact_mean8(img):
    s = int(img.reshape(-1, 4)[:, :3].astype(np.int64).sum())
    return float(Fraction(s, 3 * (img.size // 4)))


@pytest.mark.gpu
def test_device_mean_luminance_rgba8():
    """Exact integer sum on the device: the mean equals the correctly rounded
    S / 3n, and the oracle's sequential f64 sum within n * 2^-53."""
    import torch

    r = R.create_renderer(64, 48, 1)
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 4, 5, 7, 255, 1000, 65537, 1_000_003):
        img = rng.integers(0, 256, (n, 4), dtype=np.uint8)
        if n == 1000:
            img[:] = 255
        d = torch.from_numpy(img).cuda()
        m = AE.mean_luminance(r, d)
        assert m == _exact_mean8(img), n
        assert m == pytest.approx(OA.mean_luminance(img), rel=1e-12, abs=0)
    out = C.c_double(-1.0)
    _lib.check(_lib.lib().pyr3_mean_luminance(r.handle, None, 0, _lib.OUT_RGBA8, C.byref(out)))
    assert out.value == 0.0
    base = torch.zeros(64, dtype=torch.uint8, device="cuda")
    rc = _lib.lib().pyr3_mean_luminance(r.handle, C.c_void_p(base.data_ptr() + 4), 2, _lib.OUT_RGBA8,
                                        C.byref(out))
    assert rc == _lib.PYR3_E_INVALID and b"aligned" in _lib.lib().pyr3_last_error()
    r.destroy()


@pytest.mark.gpu
def test_device_mean_luminance_rgba32f_reads_as_half():
    """rgba32f: binary16 rounding (nearest even), NaN / +-inf -> 0, clamp to
    [0, 1] -- the oracle's computeMeanLuminanceHalf of the rounded image."""
    import torch

    r = R.create_renderer(64, 48, 1)
    rng = np.random.default_rng(6)
    special = np.array([np.nan, np.inf, -np.inf, -0.0, -1e-3, 1.0, 1.0001, 0.99999, 65504.0, 65519.0,
                        65520.0, 1e9, 6e-8, 3e-8, 2.9e-8, 1e-7, 0.5 + 2 ** -12, 0.5 + 3 * 2 ** -12],
                       np.float32)
    for n in (1, 6, 1000, 262_147):
        img = rng.uniform(-0.2, 1.3, (n, 4)).astype(np.float32)
        img.reshape(-1)[: min(img.size, len(special))] = special[: min(img.size, len(special))]
        m = AE.mean_luminance(r, torch.from_numpy(img).cuda())
        assert m == pytest.approx(OA.mean_luminance_rgba32f(img), rel=1e-12, abs=1e-300), n
    r.destroy()


def _render_plain(W=320, H=240):
    g = workloads.plain_small()
    g.scale = W / 4
    r = R.create_renderer(W, H, 1)
    walkers, iters, samples = R.compute_dispatch(20, W, H)
    r.reset(g)
    r.iterate(g, seed=3, walkers=walkers, iters_per_walker=iters)
    return g, r, samples


def _host_present(r, g, samples, brightness, fmt="rgba8"):
    h = copy.deepcopy(g)
    h.tonemap = dict(h.tonemap, brightness=float(np.float32(brightness)))
    return r.present(h, samples, fmt=fmt)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["rgba8", "f32", "f16"])
@pytest.mark.parametrize("ratio", [2.5, 0.3, 1.05, 0.0])
def test_device_auto_exposure_matches_oracle_loop(fmt, ratio):
    """pyr3_auto_exposure (present, device luminance, fit; 8 bytes read back
    per pass) against the oracle's fit loop over host presents.  Two
    presents of one histogram need not agree bit for bit: density
    estimation adds the discs of a tile with shared-memory float atomics in
    no fixed order, and the host presents take the brightness as f32 while
    the device loop derives k1 from the f64 brightness, as the reference
    does.  So means agree to 1e-5, brightnesses to 1e-5, f32 images to 1e-5,
    f16 images to one binary16 step and rgba8 images to one 8-bit step on
    fewer than 0.1 % of the bytes."""
    g, r, samples = _render_plain()
    base = g.tonemap["brightness"]
    measure = {"rgba8": OA.mean_luminance, "f32": OA.mean_luminance_rgba32f,
               "f16": OA.mean_luminance_half}[fmt]
    m0 = measure(_host_present(r, g, samples, base, fmt))
    target = m0 * ratio
    ref, seq = OA.fit_brightness_to_target(base, target, m0,
                                           lambda b: measure(_host_present(r, g, samples, b, fmt)))
    fit, img = AE.auto_expose(r, g, samples, target, fmt=fmt)
    assert (fit.corrected, fit.iters) == (ref[1], ref[2])
    assert fit.brightness == pytest.approx(ref[0], rel=1e-5)
    assert fit.factor == pytest.approx(ref[4], rel=1e-5)
    assert fit.final_mean == pytest.approx(ref[3], rel=1e-5)
    host = _host_present(r, g, samples, fit.brightness, fmt)
    dev = img.cpu().numpy()
    if not fit.corrected:
        assert fit.brightness == base
    if fmt == "rgba8":
        diff = np.abs(dev.astype(np.int16) - host.astype(np.int16))
        assert diff.max() <= 1 and (diff > 0).mean() < 1e-3
    elif fmt == "f32":
        assert np.allclose(dev, host, rtol=0, atol=1e-5, equal_nan=True)
    else:  # one binary16 step near 1
        assert np.allclose(dev.astype(np.float32), host.astype(np.float32), rtol=0, atol=2.0 ** -10,
                           equal_nan=True)
    if ratio in (2.5, 0.3):
        assert fit.corrected and (abs(fit.final_mean / target - 1) <= OA.AE_DEADBAND
                                  or fit.iters == OA.AE_MAX_ITERS)
    r.destroy()


@pytest.mark.gpu
def test_probe_luminance_matches_host_render():
    """measureProbeLuminance: the probe geometry, fixed seed and device mean
    equal a host render of the same probe measured by the oracle.  The two
    renders give the same histogram bit for bit; density estimation adds
    its discs with shared-memory float atomics, so the two presents may
    differ in the last f32 bit of a few pixels, which can move one 8-bit
    value: the means agree to 1e-6 (one step in ~10^5 pixel channels)."""
    g = workloads.plain_small()
    target = AE.measure_probe_luminance(g)
    probe = AE.apply_probe_preset(g)
    assert probe.size == (1024, 768) and probe.quality == 16
    r = R.create_renderer(1024, 768, 1)
    img = r.render(probe, seed=AE.AE_PROBE_SEED)
    assert target == pytest.approx(OA.mean_luminance(img), rel=1e-6)
    assert target == pytest.approx(_exact_mean8(img), rel=1e-6)
    r.destroy()


def test_fit_brightness_returns_the_callback_error_code():
    """pyr3_fit_brightness (host logic): a rerender callback that fails
    ends the fit after its first call and its code is returned, with a
    message; a null callback is refused."""
    calls = []

    def failing(b, mean_p, ctx):
        calls.append(b)
        return -7

    fn = _lib.RERENDER_FN(failing)
    out = _lib.BrightnessFit()
    rc = _lib.lib().pyr3_fit_brightness(1.0, 80.0, 10.0, fn, None, C.byref(out))
    assert rc == -7 and calls == [8.0]
    assert b"rerender" in _lib.lib().pyr3_last_error()
    rc = _lib.lib().pyr3_fit_brightness(1.0, 80.0, 10.0, _lib.RERENDER_FN(0), None, C.byref(out))
    assert rc == _lib.PYR3_E_INVALID


def test_probe_preset_scales_output_pixel_radii():
    """scaleOutputPixelRadii under force mode (src/presets.test.ts:202-275):
    DE radii and the spatial-filter radius scale with the size, the curve
    does not; sizeScale 1 leaves them untouched; no density is safe; the
    input genome is not changed."""
    g = G.Genome(scale=100.0, size=(1280, 720), quality=500,
                 density={"maxRad": 9.0, "minRad": 1.5, "curve": 0.4}, filter_radius=2.0)
    before = copy.deepcopy(g)
    out = AE.apply_probe_preset(g, 3840, 200)  # 3840 / 1280 = 3
    assert out.scale == pytest.approx(300, abs=1e-6)
    assert out.density["maxRad"] == pytest.approx(27, abs=1e-6)
    assert out.density["minRad"] == pytest.approx(4.5, abs=1e-6) and out.density["curve"] == 0.4
    assert out.filter_radius == pytest.approx(6, abs=1e-6)
    assert g == before
    same = AE.apply_probe_preset(g, 1280, 200)  # sizeScale 1
    assert same.scale == 100 and same.density == g.density and same.filter_radius == 2.0
    bare = AE.apply_probe_preset(G.Genome(scale=100.0, size=(1280, 720)), 3840, 200)
    assert bare.density is None and bare.filter_radius is None
