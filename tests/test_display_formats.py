"""Display export formats (src/gpu-readback.ts:83-115, src/srgb.ts,
src/half-float.ts): the rgba16float texture, its png16 quantisation and its
EXR linear-light transform, written on the device by the tonemap pass
(PYR3_OUT_RGBA16F / PNG16 / EXR_DISPLAY) and by pyr3_convert_display.

CPU: the oracle against the reference's own test cases.  GPU: every one
of the 65,536 binary16 patterns through pyr3_convert_display against the
oracle, f32 inputs that need rounding, and a present in every kind against
the oracle's transforms of the same present's f32 output."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import auto_exposure as OA
from oracle import display_formats as OD
from pyr3_b200 import _lib, renderer as R, workloads

H0, H1, HHALF, HNAN = 0x0000, 0x3C00, 0x3800, 0x7E00


# ---------------------------------------------------------------- CPU

def test_half_to_float_reference_cases():
    """src/half-float.test.ts."""
    f = OD.half_to_float([0x0000, 0x3C00, 0x4000, 0xC000, 0x3800, 0x0001, 0x7BFF, 0x7C00, 0xFC00])
    assert list(f[:5]) == [0.0, 1.0, 2.0, -2.0, 0.5]
    assert f[5] == pytest.approx(5.9604645e-8, abs=1e-12)
    assert f[6] == 65504.0 and f[7] == math.inf and f[8] == -math.inf
    assert math.isnan(OD.half_to_float([0x7E00])[0])
    # agrees with numpy's binary16 decoding on every pattern
    allb = np.arange(65536, dtype=np.uint32)
    ref = allb.astype(np.uint16).view(np.float16).astype(np.float64)
    got = OD.half_to_float(allb)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    assert np.array_equal(got[~np.isnan(got)], ref[~np.isnan(ref)])


def test_srgb_to_linear_reference_cases():
    """src/srgb.test.ts."""
    s = OD.srgb_to_linear([0.0, 1.0, 0.5, 0.04045, 0.02])
    assert s[0] == 0 and s[1] == pytest.approx(1, abs=1e-6) and s[2] == pytest.approx(0.21404, abs=1e-4)
    assert s[3] == pytest.approx(0.04045 / 12.92, abs=1e-7) and s[4] == pytest.approx(0.02 / 12.92, abs=1e-7)


def test_display_transforms_reference_cases():
    """src/gpu-readback.test.ts:40-72."""
    exr = OD.display_half_to_linear_exr([H1, H0, HHALF, HHALF])[0]
    assert exr[0] == pytest.approx(OD.srgb_to_linear(1.0), abs=1e-6)
    assert exr[1] == pytest.approx(OD.srgb_to_linear(0.0), abs=1e-6)
    assert exr[2] == pytest.approx(OD.srgb_to_linear(0.5), abs=1e-6)
    assert exr[3] == pytest.approx(0.5, abs=1e-6)
    assert list(OD.display_half_to_linear_exr([HNAN] * 4)[0]) == [0, 0, 0, 0]
    neg0 = OD.display_half_to_linear_exr([0x8000] * 4)[0]  # -0 clamps to +0 (JS Math.max)
    assert not np.signbit(neg0).any()
    png = OD.display_half_to_png16([H1, H0, HHALF, H1])[0]
    assert list(png) == [65535, 0, math.floor(0.5 * 65535 + 0.5), 65535]
    assert list(OD.display_half_to_png16([HNAN] * 4)[0]) == [0, 0, 0, 0]


# ---------------------------------------------------------------- GPU

def _convert(src_f32: np.ndarray, kind: int, dtype):
    import torch

    d_in = torch.from_numpy(np.ascontiguousarray(src_f32, np.float32).reshape(-1, 4)).cuda()
    d_out = torch.empty((d_in.shape[0], 4), dtype=dtype, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().pyr3_convert_display(C.c_void_p(d_in.data_ptr()), d_in.shape[0], kind,
                                               C.c_void_p(d_out.data_ptr()), None))
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


def _f32_ulps(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ai = a.astype(np.float32).view(np.int32).astype(np.int64)
    bi = b.astype(np.float32).view(np.int32).astype(np.int64)
    return np.abs(ai - bi)


def _inputs():
    """Every binary16 pattern (as its exact f32 value) plus f32 values that
    need rounding: random in [-0.5, 1.5], halfway cases, overflow,
    subnormal halves."""
    allh = np.arange(65536, dtype=np.uint32).astype(np.uint16).view(np.float16).astype(np.float32)
    rng = np.random.default_rng(17)
    extra = np.concatenate([rng.uniform(-0.5, 1.5, 40_000).astype(np.float32),
                            np.float32(0.5) + np.float32(2.0 ** -12) * np.arange(1, 64, 2, dtype=np.float32),
                            np.array([65519, 65520, 1e9, -1e9, 3e-8, 2.9e-8, 6e-8, 1e-45], np.float32)])
    x = np.concatenate([allh, extra])
    return np.concatenate([x, np.zeros((-len(x)) % 4, np.float32)])


@pytest.mark.gpu
def test_convert_display_every_half_pattern():
    x = _inputs()
    bits = OD.to_half_bits(x)
    f16 = _convert(x, _lib.OUT_RGBA16F, __import__("torch").float16).reshape(-1).view(np.uint16)
    nan = np.isnan(bits.view(np.float16))
    assert np.array_equal(np.isnan(f16.view(np.float16)), nan)
    assert np.array_equal(f16[~nan], bits[~nan])
    png = _convert(x, _lib.OUT_PNG16, __import__("torch").int16).reshape(-1).view(np.uint16)
    assert np.array_equal(png, OD.display_half_to_png16(bits).reshape(-1))
    exr = _convert(x, _lib.OUT_EXR_DISPLAY, __import__("torch").float32).reshape(-1)
    ref = OD.display_half_to_linear_exr(bits).reshape(-1)
    ulps = _f32_ulps(exr, ref)
    print(f"exr: {int((ulps > 0).sum())} of {len(ulps)} values differ from the oracle (max {int(ulps.max())} ulp)")
    assert int(ulps.max()) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("os_", [1, 2])
def test_present_in_every_kind_matches_the_oracle_transforms(os_):
    """One histogram (density estimation off, so every present is the same
    bit for bit) presented as f32, f16, png16 and exr: f16 is the f32
    present rounded to binary16, and png16 / exr are the oracle's transforms
    of that f16 image."""
    W, H = 96, 64
    g = workloads.plain_small()
    g.scale = W / 4
    r = R.create_renderer(W, H, os_)
    walkers, iters, samples = R.compute_dispatch(30, W, H)
    r.reset(g)
    r.iterate(g, seed=9, walkers=walkers, iters_per_walker=iters)
    f32 = r.present(g, samples, force_de_off=True, fmt="f32")
    f16 = r.present(g, samples, force_de_off=True, fmt="f16")
    bits = OD.to_half_bits(f32)
    assert np.array_equal(f16.view(np.uint16), bits)
    png = r.present(g, samples, force_de_off=True, fmt="png16")
    assert np.array_equal(png.reshape(-1, 4), OD.display_half_to_png16(bits))
    exr = r.present(g, samples, force_de_off=True, fmt="exr")
    assert int(_f32_ulps(exr.reshape(-1, 4), OD.display_half_to_linear_exr(bits)).max()) == 0
    r.destroy()


@pytest.mark.gpu
def test_mean_luminance_of_the_half_texture():
    """computeMeanLuminanceHalf of an rgba16f device image (ragged pixel
    counts, NaN / inf patterns) against the oracle."""
    import torch

    from pyr3_b200 import auto_exposure as AE

    r = R.create_renderer(16, 16, 1)
    rng = np.random.default_rng(4)
    for n in (1, 3, 1001, 65_537):
        bits = rng.integers(0, 65536, (n, 4)).astype(np.uint16)
        bits[::7, 0] = 0x7E00
        bits[::11, 1] = 0x7C00
        img = torch.from_numpy(bits.view(np.float16)).cuda()
        m = AE.mean_luminance(r, img)
        assert m == pytest.approx(OA.mean_luminance_half(bits.view(np.float16)), rel=1e-12, abs=1e-300), n
    r.destroy()


def test_present_formats_map_to_the_c_abi_kinds():
    """Renderer.present's format names, the PYR3_OUT_* kinds and their host
    element types (host logic, no GPU)."""
    import re

    hdr = open(__import__("os").path.join(__import__("os").path.dirname(__file__), "..", "include",
                                          "pyr3.h")).read()
    kinds = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define PYR3_OUT_(\w+) (\d+)", hdr)}
    assert kinds == {"RGBA8": 0, "RGBA32F": 1, "RGBA16F": 2, "PNG16": 3, "EXR_DISPLAY": 4}
    assert {k: v[0] for k, v in R.FORMATS.items()} == {"rgba8": 0, "f32": 1, "f16": 2, "png16": 3, "exr": 4}
    assert [np.dtype(v[1]).itemsize * 4 for v in R.FORMATS.values()] == [4, 16, 8, 8, 16]


def test_convert_display_refuses_bad_arguments():
    """pyr3_convert_display checks its kind and alignment before any device
    work (host logic): an unknown kind and misaligned buffers are refused;
    zero pixels is a no-op."""
    buf = (C.c_uint8 * 64)()
    base = C.addressof(buf)
    aligned = base + (-base) % 16
    L = _lib.lib()
    assert L.pyr3_convert_display(C.c_void_p(aligned), 1, 9, C.c_void_p(aligned), None) == _lib.PYR3_E_INVALID
    assert L.pyr3_convert_display(C.c_void_p(aligned + 4), 1, _lib.OUT_PNG16, C.c_void_p(aligned),
                                  None) == _lib.PYR3_E_INVALID
    assert b"aligned" in L.pyr3_last_error()
    assert L.pyr3_convert_display(C.c_void_p(aligned), 1, _lib.OUT_PNG16, C.c_void_p(aligned + 8),
                                  None) == _lib.PYR3_E_INVALID
    assert L.pyr3_convert_display(None, 0, _lib.OUT_EXR_DISPLAY, None, None) == _lib.PYR3_OK
