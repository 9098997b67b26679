"""GPU: whole renders of the benchmark genomes against the reference's own
chaos loop (chaos_main, src/shaders/chaos.wgsl:8269-8731, translated for
the CPU) at equal sample count.

Trajectories diverge chaotically under one-ulp differences of the catalog
variations, so the comparison is statistical, on two measures:

* log-density relative L1 (log1p of each output pixel's count / 255, summed
  over the oversample block) at most 1 % or 1.5x the reference-vs-
  reference floor (the same render at another seed);
* the tonemapped image (the oracle's density estimation and visualize of the
  reference histogram, the device present of the CUDA one): PSNR at least
  40 dB, or within 1 dB of the reference-vs-reference PSNR where two
  reference seeds are themselves closer than 40 dB.

The genomes are the benchmark's own (pyr3_b200/workloads.py) on reduced
canvases at the benchmark's samples per pixel: the headline genome (12
catalog xforms, post affines, final xform) through the wave kernel at the
bench's ~3,077 iterations per walker and at the short-trajectory pool of a
small launch; the motion_4k genome (direct-colour variations, 8 box-
filtered sub-frames, density estimation 15/0/0.6 at oversample 2, radius
31); and eight batch_256 genomes through one batch."""
import copy

import numpy as np
import pytest

from oracle import oracle as O
from pyr3_b200 import animate as A
from pyr3_b200 import renderer as R
from pyr3_b200 import workloads
from pyr3_b200.genome import DEFAULT_TONEMAP
from refrender import THREADS, chaos as ref_chaos, log_density_l1, psnr

pytestmark = pytest.mark.gpu


def _tonemapped_ref(g, hist, W, H, os_, samples):
    """The oracle's present of a reference histogram: density estimation
    (when the genome sets it) and visualize, RGB in [0, 1]."""
    tm = dict(DEFAULT_TONEMAP)
    tm.update(g.tonemap or {})
    k1, k2 = O.derive_calibration(g.scale, samples, tm["brightness"], os_)
    src = {}
    if g.density:
        de = g.density
        src["src_f32"] = O.ref_density(hist, W * os_, H * os_, de["maxRad"] * os_ + 1,
                                       de["minRad"] * os_ + 1, de["curve"], np.float32(k1), np.float32(k2),
                                       threads=THREADS)
    else:
        src["src_u32"] = hist
    img = O.visualize(W, H, os_, O.spatial_kernel(0.5, os_), np.float32(k1), np.float32(k2), tm["gamma"],
                      tm["vibrancy"], tm["highlightPower"], tm["gammaThreshold"], **src)
    return img.reshape(H, W, 4)[..., :3].astype(np.float64)


def _check(name, g, dev_hist, dev_img, ref1, ref2, W, H, os_, samples):
    l1 = log_density_l1(dev_hist, ref1, W, H, os_)
    floor = log_density_l1(ref2, ref1, W, H, os_)
    i1 = _tonemapped_ref(g, ref1, W, H, os_, samples)
    i2 = _tonemapped_ref(g, ref2, W, H, os_, samples)
    p_dev, p_floor = psnr(dev_img, i1), psnr(i2, i1)
    print(f"{name}: log-density L1 {l1:.3%} (ref-vs-ref {floor:.3%}); "
          f"PSNR {p_dev:.2f} dB (ref-vs-ref {p_floor:.2f} dB)")
    assert l1 <= max(0.01, 1.5 * floor), (l1, floor)
    assert p_dev >= min(40.0, p_floor - 1.0), (p_dev, p_floor)
    return l1, floor, p_dev, p_floor


# Iterations per walker of the bench's headline launch: 1.0368e9 samples on
# ~338,000 walkers (the wave pool whose records fill half of L2: 337,920 on
# B200, ~3,068 iterations each; 3,077 is within 0.3 % of that).
BENCH_ITERS = 3077


@pytest.mark.parametrize("pool,W,H,spp", [("bench_iters", 480, 270, 500),
                                          ("short_trajectories", 480, 270, 500),
                                          ("bench_iters", 192, 108, 6000)])
def test_headline_genome_matches_reference(pool, W, H, spp):
    """The headline genome (1920x1080 os 2, 500 spp, 12 catalog xforms +
    final) on reduced os-2 canvases through the wave kernel, against the
    reference's computeDispatch split (1024 walkers):

    * 480x270 at the bench's 500 spp (6.48e7 samples), with walkers of 3,077
      iterations (about the bench's iterations per walker: ~338,000 walkers at full
      size), and with the small-launch pool (~279k walkers of ~232
      iterations, where the 200-iteration burn-in weighs most).  At 500 spp
      two reference seeds are themselves only ~32.6 dB apart, so the image
      bar is the reference-vs-reference PSNR less 1 dB;
    * 192x108 at 6,000 spp (1.24e8 samples), where the reference-vs-
      reference floor is above 40 dB: the device render is at least 40 dB
      from the reference.

    With 3,077-iteration walkers the device draws samples // 3077 x 3077
    samples (at most 3,076 fewer than the reference), and each image is
    presented with its own sample count."""
    g = workloads.headline_1080p()
    os_ = 2
    g.scale = W / 4
    walkers, iters, samples = R.compute_dispatch(spp, W, H)
    ref1 = ref_chaos(g, W * os_, H * os_, iters, walkers, seed=9, oversample=os_)
    ref2 = ref_chaos(g, W * os_, H * os_, iters, walkers, seed=31, oversample=os_)
    r = R.create_renderer(W, H, os_)
    r.reset(g)
    if pool == "bench_iters":
        dev_samples = samples // BENCH_ITERS * BENCH_ITERS
        r.iterate(g, seed=77, walkers=dev_samples // BENCH_ITERS, iters_per_walker=BENCH_ITERS, exact_walkers=True,
                  kernel="wave")
    else:
        dev_samples = samples
        r.iterate(g, seed=77, walkers=walkers, iters_per_walker=iters, kernel="wave")
    assert r.counters()[0] == dev_samples
    dev, _, _ = r.read_histogram()
    img = r.present(g, dev_samples, fmt="f32")[..., :3].astype(np.float64)
    r.destroy()
    _, _, p_dev, p_floor = _check(f"headline/{pool}/{W}x{H}/{spp}spp", g, dev.reshape(-1), img, ref1, ref2,
                                  W, H, os_, samples)
    if spp >= 6000:
        assert p_floor >= 40.0 and p_dev >= 40.0, (p_dev, p_floor)


def test_motion_4k_genome_matches_reference_subframe_loop():
    """The motion_4k genome (6 xforms mixing flam3-core and direct-colour
    variations, affines interpolated across the shutter) as one motion-
    blurred frame of 8 box-filtered sub-frames on a 320x180 os-2 canvas at
    400 spp, with density estimation 15/0/0.6 (radius 31 at oversample 2):
    render_motion_frame against the reference's chaos_main run for every
    sub-frame genome with the same walker split and seeds
    (src/animate-render.ts:95-168), each histogram presented by the
    oracle's density estimation and visualize."""
    g0, g1 = workloads.motion_4k()
    W, H, os_ = 320, 180, 2
    for g in (g0, g1):
        g.scale = W / 4
        g.quality = 400
    walkers, iters, samples = R.compute_dispatch(400, W, H)
    deltas, filt, _ = A.temporal_filter(8)
    counts = A.apportion_walkers(walkers, filt)

    def ref(seed):
        hist = np.zeros(W * os_ * H * os_ * 4, np.uint32)
        for i, w in enumerate(counts):
            sub = A.interpolate_linear(g0, g1, 0.5 + deltas[i])
            ref_chaos(sub, W * os_, H * os_, iters, w, (seed + i * A.GOLDEN) & 0xFFFFFFFF,
                      oversample=os_, hist=hist)
        return hist

    ref1, ref2 = ref(9), ref(31)
    r = R.create_renderer(W, H, os_)
    n, c = A.render_motion_frame(r, g0, g1, 0.5, ntemporal=8, seed=77)
    assert n == samples and sum(c) == walkers
    dev, _, _ = r.read_histogram()
    centre = A.interpolate_linear(g0, g1, 0.5)
    img = r.present(centre, samples, fmt="f32")[..., :3].astype(np.float64)
    r.destroy()
    _check("motion_4k", centre, dev.reshape(-1), img, ref1, ref2, W, H, os_, samples)


def test_batch_genomes_match_reference():
    """Eight batch_256 genomes (2-20 xforms of 1-6 catalog variations) on
    200x150 canvases at 300 spp, rendered together by one batch (per-genome
    walker plans, one graph): every genome against the reference's
    chaos_main at its computeDispatch split."""
    from pyr3_b200 import batch as B

    W, H = 200, 150
    gs = []
    for g in workloads.batch_256()[:8]:
        g = copy.deepcopy(g)
        g.size = (W, H)
        g.scale = W / 4
        g.quality = 300.0
        g.density = None
        gs.append(g)
    b = B.Batch(gs, n_streams=4, seed=5)
    b.run()
    b.sync()
    worst = []
    for i, g in enumerate(gs):
        walkers, iters, samples = R.compute_dispatch(g.quality, W, H)
        assert b.renderers[i].counters()[0] == b.samples[i] == samples
        dev, _, _ = b.renderers[i].read_histogram()
        img = b.present(i, fmt="f32")[..., :3].astype(np.float64)
        ref1 = ref_chaos(g, W, H, iters, walkers, seed=9)
        ref2 = ref_chaos(g, W, H, iters, walkers, seed=31)
        worst.append(_check(f"batch genome {i} ({len(g.xforms)} xforms)", g, dev.reshape(-1), img, ref1,
                            ref2, W, H, 1, samples))
    b.destroy()
