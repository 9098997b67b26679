"""GPU: the allocation-free present, pyr3_density_tonemap_noalloc.

It serves callers that cannot allocate device memory (code running inside
another engine's frame loop or memory pool, or code that must not allocate
once it is running): they hand over a histogram already on the device and
an output image on the device, and the library does density estimation and
tonemap in a fixed scratch array of its own.  Here it must give the same
image as the allocating entry point pyr3_density_tonemap on the same
histogram, on two calls in a row (so the second call sees the first call's
leftovers in the shared array), and it must refuse canvases larger than its
fixed scratch.

The device buffers below are the test's own (torch); the entry point under
test allocates nothing, which the tests also check against the device's free
memory.  This file is collected last on purpose.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from pyr3_b200 import _lib, renderer as R, workloads

pytestmark = pytest.mark.gpu

TOL = 1.0 / 255.0  # the tolerance of the density + tonemap parity tests


def _histogram(W, H, os_, seed):
    """A seeded super-res histogram shaped like a render: a blob of hits,
    count channel 255 per hit, colour channels up to the count."""
    rng = np.random.default_rng(seed)
    sw, sh = W * os_, H * os_
    yy, xx = np.mgrid[0:sh, 0:sw]
    lam = 40.0 * np.exp(-(((xx - sw * 0.45) / (0.2 * sw)) ** 2 + ((yy - sh * 0.55) / (0.25 * sh)) ** 2))
    hits = rng.poisson(lam).astype(np.uint64)
    hist = np.zeros((sh, sw, 4), np.uint32)
    hist[..., 3] = (hits * 255).astype(np.uint32)
    for c in range(3):
        hist[..., c] = (hist[..., 3] * rng.uniform(0.0, 1.0, (sh, sw))).astype(np.uint32)
    return hist.reshape(-1), int(hits.sum())


def _present_opts(W, de_on, max_rad, curves=False):
    g = workloads.plain_small()
    g.scale = W / 4
    g.density = {"maxRad": max_rad, "minRad": 0.0, "curve": 0.4}
    if curves:
        g.channel_curves = {"composite": [(0, 0.05), (0.5, 0.6), (1, 1)], "g": [(0, 0.1), (1, 0.8)],
                            "luma": [(0, 0), (0.4, 0.5), (1, 1)]}
    return R.Renderer.present_opts(None, g, force_de_off=not de_on)


def _allocating(hist, W, H, os_, p, samples):
    out = np.zeros(W * H * 4, np.float32)
    _lib.check(_lib.lib().pyr3_density_tonemap(_lib.ptr(hist), W, H, os_, 0.5, C.byref(p), samples,
                                               _lib.ptr(out), None))
    return out


def _no_alloc(hist, W, H, os_, p, samples, kind=None):
    import torch

    kind = _lib.OUT_RGBA32F if kind is None else kind
    d_hist = torch.from_numpy(hist.view(np.int32)).cuda()
    if kind == _lib.OUT_RGBA8:
        d_out = torch.zeros(W * H * 4, dtype=torch.uint8, device="cuda")
    else:
        d_out = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().pyr3_density_tonemap_noalloc(
        C.c_void_p(d_hist.data_ptr()), W, H, os_, 0.5, C.byref(p), samples,
        C.c_void_p(d_out.data_ptr()), kind, C.c_void_p(stream)))
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


def test_no_alloc_present_matches_allocating_present_twice():
    """Two calls in a row, a larger canvas with density estimation first,
    then a smaller one with another radius: each equals
    pyr3_density_tonemap within 1/255 per channel."""
    cases = [(200, 150, 2, True, 9.0, 11), (160, 120, 1, True, 15.0, 12)]
    for W, H, os_, de_on, max_rad, seed in cases:
        hist, samples = _histogram(W, H, os_, seed)
        p = _present_opts(W, de_on, max_rad)
        want = _allocating(hist, W, H, os_, p, samples)
        got = _no_alloc(hist, W, H, os_, p, samples)
        assert float(np.abs(got - want).max()) <= TOL, (W, H, os_)
        assert float(want[3::4].max()) > 0.0


def test_no_alloc_present_refuses_oversized_canvas():
    """1024 x 1024 at oversample 2 needs 4 Mi super-sampled pixels, more
    than the fixed scratch holds: a clear error, nothing launched."""
    import torch

    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = _present_opts(1024, True, 9.0)
    rc = _lib.lib().pyr3_density_tonemap_noalloc(C.c_void_p(d.data_ptr()), 1024, 1024, 2, 0.5,
                                                 C.byref(p), 1000, C.c_void_p(d.data_ptr()),
                                                 _lib.OUT_RGBA32F, None)
    assert rc != 0
    assert "super-sampled pixels" in _lib.lib().pyr3_last_error().decode()


def test_no_alloc_present_without_density_with_curves_and_rgba8():
    """Density estimation off (the tonemap reads the caller's histogram
    directly) with colour curves on, in the f32 kind and in rgba8: equal to
    the allocating present within 1/255 (rgba8: within one 8-bit step of
    its rounding of the f32 image)."""
    W, H, os_ = 180, 120, 2
    hist, samples = _histogram(W, H, os_, 21)
    p = _present_opts(W, False, 9.0, curves=True)
    assert p.curves_active != 0 and p.density_on == 0
    want = _allocating(hist, W, H, os_, p, samples)
    got = _no_alloc(hist, W, H, os_, p, samples)
    assert float(np.abs(got - want).max()) <= TOL
    got8 = _no_alloc(hist, W, H, os_, p, samples, kind=_lib.OUT_RGBA8).astype(np.int32)
    want8 = np.rint(np.clip(want, 0.0, 1.0) * 255.0).astype(np.int32)
    assert int(np.abs(got8 - want8).max()) <= 1
    assert int(got8[0::4].max()) > 0


def test_no_alloc_present_leaves_free_device_memory_unchanged():
    """After a first call (set-up done, kernels loaded), a second identical
    call leaves the device's free memory as it was: the entry point
    allocates nothing."""
    import torch

    W, H, os_ = 200, 150, 2
    hist, samples = _histogram(W, H, os_, 31)
    p = _present_opts(W, True, 9.0)
    d_hist = torch.from_numpy(hist.view(np.int32)).cuda()
    d_out = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        _lib.check(_lib.lib().pyr3_density_tonemap_noalloc(
            C.c_void_p(d_hist.data_ptr()), W, H, os_, 0.5, C.byref(p), samples,
            C.c_void_p(d_out.data_ptr()), _lib.OUT_RGBA32F, stream))
        torch.cuda.synchronize()

    call()
    free0 = torch.cuda.mem_get_info()[0]
    call()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    assert float(d_out[3::4].max()) > 0.0


_FRESH = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import test_zz_no_alloc as T
from pyr3_b200 import _lib
W, H, os_ = 160, 120, 2
hist, samples = T._histogram(W, H, os_, 41)
p = T._present_opts(W, True, 9.0)
want = T._allocating(hist, W, H, os_, p, samples)
s = torch.cuda.Stream()
with torch.cuda.stream(s):
    d_hist = torch.from_numpy(hist.view(np.int32)).cuda()
    d_out = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().pyr3_density_tonemap_noalloc(
        C.c_void_p(d_hist.data_ptr()), W, H, os_, 0.5, C.byref(p), samples,
        C.c_void_p(d_out.data_ptr()), _lib.OUT_RGBA32F, C.c_void_p(s.cuda_stream)))
s.synchronize()
got = d_out.cpu().numpy()
err = float(np.abs(got - want).max())
assert err <= T.TOL, err
print("fresh-process first call on a non-blocking stream: max err", err)
"""


def test_no_alloc_first_call_on_a_non_blocking_stream_in_a_fresh_process():
    """The first call of a process sets the fixed array up on the caller's
    stream.  In a fresh process whose first call runs on a torch stream
    (created non-blocking, so it does not wait for the legacy default
    stream), the image still equals the allocating present within 1/255."""
    import torch

    assert torch.cuda.Stream().cuda_stream != 0
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    print(r.stdout.strip())

