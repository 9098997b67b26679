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
test allocates nothing.  This file is collected last on purpose.
"""
import ctypes as C

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


def _present_opts(W, de_on, max_rad):
    g = workloads.plain_small()
    g.scale = W / 4
    g.density = {"maxRad": max_rad, "minRad": 0.0, "curve": 0.4}
    return R.Renderer.present_opts(None, g, force_de_off=not de_on)


def _allocating(hist, W, H, os_, p, samples):
    out = np.zeros(W * H * 4, np.float32)
    _lib.check(_lib.lib().pyr3_density_tonemap(_lib.ptr(hist), W, H, os_, 0.5, C.byref(p), samples,
                                               _lib.ptr(out), None))
    return out


def _no_alloc(hist, W, H, os_, p, samples):
    import torch

    d_hist = torch.from_numpy(hist.view(np.int32)).cuda()
    d_out = torch.zeros(W * H * 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().pyr3_density_tonemap_noalloc(
        C.c_void_p(d_hist.data_ptr()), W, H, os_, 0.5, C.byref(p), samples,
        C.c_void_p(d_out.data_ptr()), _lib.OUT_RGBA32F, C.c_void_p(stream)))
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
