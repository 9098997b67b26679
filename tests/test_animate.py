"""Motion-blurred frames (src/temporal-filter.ts, src/animate-render.ts,
src/interpolate.ts): CPU checks restating the reference's own test cases
(src/temporal-filter.test.ts, src/animate-render.test.ts), and a GPU check of
a whole motion-blurred frame against the reference's chaos loop run per
sub-frame."""
import copy

import numpy as np
import pytest

from pyr3_b200 import animate as A
from pyr3_b200 import workloads


def test_temporal_filter_matches_reference_cases():
    assert A.temporal_filter(1, "box", 1.0, 0) == ([0.0], [1.0], 1.0)
    d, f, s = A.temporal_filter(4, "box", 1.0, 0)
    assert d[0] == pytest.approx(-0.5) and d[3] == pytest.approx(0.5)
    assert d[1] - d[0] == pytest.approx(1 / 3)
    assert f == [1, 1, 1, 1] and s == pytest.approx(1.0)
    d, _, _ = A.temporal_filter(4, "box", 2.0, 0)
    assert d[0] == pytest.approx(-1) and d[3] == pytest.approx(1)
    _, f, s = A.temporal_filter(11, "gaussian", 1.0, 0)
    assert f[5] > f[0] and max(f) == pytest.approx(1.0) and 0 < s < 1
    _, f, _ = A.temporal_filter(10, "exp", 1.0, 2.0)
    assert f[9] == pytest.approx(1.0) and f[0] < f[9]
    _, f, _ = A.temporal_filter(10, "exp", 1.0, -2.0)
    assert f[0] == pytest.approx(1.0) and f[9] < f[0]
    _, f, _ = A.temporal_filter(10, "exp", 1.0, 0.0)
    assert all(v == pytest.approx(1.0) for v in f)


def test_apportion_walkers_matches_reference_cases():
    out = A.apportion_walkers(1024, [1] * 2000)
    assert sum(out) == 1024 and sum(1 for w in out if w == 0) > 900
    out = A.apportion_walkers(100, [0.05, 0.3, 1.0, 0.3, 0.05])
    assert sum(out) == 100 and out[2] > out[1] and out[2] > out[3]
    assert A.apportion_walkers(64, [0, 0, 1, 0]) == [0, 0, 64, 0]
    assert A.apportion_walkers(0, [1, 1, 1]) == [0, 0, 0]
    assert A.apportion_walkers(100, [0, 0]) == [0, 0]
    assert A.apportion_walkers(100, []) == []
    for n in (3, 7, 1000, 4096):
        out = A.apportion_walkers(1024, [1] * n)
        assert sum(out) == 1024 and min(out) >= 0


def test_interpolate_linear_endpoints_and_midpoint():
    g0, g1 = workloads.motion_4k()
    a = A.interpolate_linear(g0, g1, 0.0)
    b = A.interpolate_linear(g0, g1, 1.0)
    m = A.interpolate_linear(g0, g1, 0.5)
    for x, x0, x1, xa, xb in zip(m.xforms, g0.xforms, g1.xforms, a.xforms, b.xforms):
        for k in "abcdef":
            assert getattr(xa, k) == pytest.approx(getattr(x0, k))
            assert getattr(xb, k) == pytest.approx(getattr(x1, k))
            assert getattr(x, k) == pytest.approx(0.5 * getattr(x0, k) + 0.5 * getattr(x1, k))
    bad = copy.deepcopy(g1)
    bad.xforms = bad.xforms[:-1]
    with pytest.raises(ValueError):
        A.interpolate_linear(g0, bad, 0.5)


def _motion_pair():
    """The C1 genome at shutter open and a copy with its affines moved."""
    g0 = workloads.plain_small()
    g1 = copy.deepcopy(g0)
    rng = np.random.default_rng(4)
    for x in g1.xforms:
        x.a, x.b, x.c, x.d, x.e, x.f = (v + float(dv) for v, dv in
                                        zip((x.a, x.b, x.c, x.d, x.e, x.f), rng.uniform(-0.08, 0.08, 6)))
    return g0, g1


@pytest.mark.gpu
def test_motion_frame_matches_reference_subframe_loop():
    """4 box-filtered sub-frames of a moving C1 genome on 160x120: the CUDA
    path (render_motion_frame) vs the reference's chaos_main (translated
    WGSL, CPU) run for each sub-frame genome with the same walker split into
    one histogram, at equal samples: log-density L1 within 1% or 1.5x the
    reference-vs-reference floor."""
    from oracle import oracle as O
    from pyr3_b200 import genome as G, renderer as R

    W, H, iters = 160, 120, 48_000
    g0, g1 = _motion_pair()
    for g in (g0, g1):
        g.scale = W / 4
        g.quality = 1024 * iters / (W * H)

    def ref(seed):
        hist = np.zeros(W * H * 4, np.uint32)
        deltas, filt, _ = A.temporal_filter(4)
        counts = A.apportion_walkers(1024, filt)
        for i, w in enumerate(counts):
            sub = A.interpolate_linear(g0, g1, 0.5 + deltas[i])
            u = np.zeros(31, np.uint32)
            f, i32 = u.view(np.float32), u.view(np.int32)
            u[0], u[1], u[2], u[3] = W, H, iters, 200
            f[4], f[5], f[6] = sub.scale, 0.0, 0.0
            u[7] = (seed + i * A.GOLDEN) & 0xFFFFFFFF
            i32[8] = -1
            u[12] = w
            f[13] = 1e-7
            O.ref_chaos_run(u, G.pack_xforms(sub), len(sub.xforms), G.bake_lut(sub.palette),
                            O.pack_xform_distrib([x.weight for x in sub.xforms]),
                            O.pack_isaac_states(w, u[7]), 0, w, hist, 16)
        return hist

    def logd(h):
        return np.log1p(h.reshape(-1, 4)[:, 3].astype(np.float64) / 255.0)

    r = R.create_renderer(W, H, 1)
    samples, counts = A.render_motion_frame(r, g0, g1, 0.5, ntemporal=4, seed=77)
    assert sum(counts) == 1024 and samples == 1024 * iters
    assert r.counters()[0] == samples
    dev, _, _ = r.read_histogram()
    a, b, b2 = logd(dev), logd(ref(9)), logd(ref(31))
    l1 = float(np.abs(a - b).sum() / b.sum())
    floor = float(np.abs(b2 - b).sum() / b.sum())
    print(f"motion log-density L1 {l1:.4%} (ref-vs-ref {floor:.4%})")
    assert l1 <= max(0.01, 1.5 * floor), (l1, floor)
    r.destroy()


def _logd(h):
    return np.log1p(h.reshape(-1, 4)[:, 3].astype(np.float64) / 255.0)


@pytest.mark.gpu
def test_animation_batch_frames_match_the_frame_loop():
    """Six frames of the moving C1 genome, 4 box sub-frames each, rendered
    by one AnimationBatch (24 genomes in one graph, 4 per renderer): every
    frame accumulates exactly its sample count, and its histogram matches
    render_motion_frame of the same frame within 1 % log-density L1 or
    1.5x the floor between two seeds of render_motion_frame."""
    from pyr3_b200 import renderer as R

    W, H = 160, 120
    g0, g1 = _motion_pair()
    for g in (g0, g1):
        g.scale = W / 4
        g.quality = 400
        g.size = (W, H)
    times = [0.2, 0.3, 0.4, 0.5, 0.6, 0.7]
    ab = A.AnimationBatch(g0, g1, times, ntemporal=4, seed=5)
    assert ab.n_genomes == 24
    ab.run()
    _, total = ab.sync()
    assert total == sum(ab.samples)
    r = R.create_renderer(W, H, 1)
    worst = []
    for k, t in enumerate(times):
        assert ab.renderers[k].counters()[0] == ab.samples[k]
        a = _logd(ab.renderers[k].read_histogram()[0])
        n1, _ = A.render_motion_frame(r, g0, g1, t, ntemporal=4, seed=9)
        b = _logd(r.read_histogram()[0])
        A.render_motion_frame(r, g0, g1, t, ntemporal=4, seed=31)
        b2 = _logd(r.read_histogram()[0])
        assert n1 == ab.samples[k]
        l1 = float(np.abs(a - b).sum() / b.sum())
        floor = float(np.abs(b2 - b).sum() / b.sum())
        worst.append((l1, floor))
        assert l1 <= max(0.01, 1.5 * floor), (k, l1, floor)
    print("frame L1 vs floor:", [f"{a:.3%}/{b:.3%}" for a, b in worst])
    img = ab.present(2)
    assert img.shape == (H, W, 4) and img[..., :3].any()
    # a second run clears and re-accumulates: the same counts again
    ab.run()
    ab.sync()
    assert [rr.counters()[0] for rr in ab.renderers] == ab.samples
    ab.destroy()
    r.destroy()


@pytest.mark.gpu
def test_animation_batch_mixes_graph_and_solo_sub_frames_in_one_frame():
    """A gaussian temporal filter splits walkers unevenly, so the middle
    sub-frames of a high-quality frame reach 2^24 samples and run through
    pyr3_iterate beside the graph while its tails run in the graph, all
    into the same histogram: the frame still counts exactly its samples."""
    W, H = 160, 120
    g0, g1 = _motion_pair()
    for g in (g0, g1):
        g.scale = W / 4
        g.quality = 4500
        g.size = (W, H)
    ab = A.AnimationBatch(g0, g1, [0.3, 0.6], ntemporal=7, filter_kind="gaussian", seed=3)
    _, reqs, total = A._frame_plan(g0, g1, 0.3, W, H, 7, "gaussian", 1.0, 0.0, 3)
    sizes = [w * it for _, _, w, it in reqs]
    assert max(sizes) >= 1 << 24 and min(sizes) < 1 << 24, sizes
    ab.run()
    ab.sync()
    assert [r.counters()[0] for r in ab.renderers] == ab.samples
    hist = ab.renderers[0].read_histogram()[0]
    assert int(hist.reshape(-1, 4)[:, 3].astype(np.uint64).sum()) == 255 * ab.renderers[0].counters()[1]
    ab.destroy()


def test_frame_plan_restates_render_animation_frame():
    """The per-frame plan AnimationBatch submits (host logic, no GPU) is
    renderAnimationFrame's (src/animate-render.ts:73-176): the centre genome
    at the frame time, walkers apportioned by the temporal filter (zero-
    weight tails dropped), every sub-frame at the centre's iterations,
    seeds base + i * 0x9e3779b1, and a total of walkers x iterations."""
    from pyr3_b200.renderer import compute_dispatch

    g0, g1 = _motion_pair()
    for g in (g0, g1):
        g.quality = 50
    W, H = 320, 180
    for n, kind in ((1, "box"), (4, "box"), (7, "gaussian"), (9, "exp")):
        centre, reqs, total = A._frame_plan(g0, g1, 0.4, W, H, n, kind, 1.0, 0.5, 1234)
        walkers, iters, _ = compute_dispatch(50, W, H)
        assert centre.xforms[0].a == A.interpolate_linear(g0, g1, 0.4).xforms[0].a
        assert all(it == iters for _, _, _, it in reqs)
        if n == 1:
            assert [(s, w) for _, s, w, _ in reqs] == [(1234, walkers)]
            continue
        deltas, filt, _ = A.temporal_filter(n, kind, 1.0, 0.5)
        counts = A.apportion_walkers(walkers, filt)
        kept = [i for i, c in enumerate(counts) if c > 0]
        assert [w for _, _, w, _ in reqs] == [counts[i] for i in kept]
        assert [s for _, s, _, _ in reqs] == [(1234 + i * A.GOLDEN) & 0xFFFFFFFF for i in kept]
        for (g, _, _, _), i in zip(reqs, kept):
            assert g.xforms[1].e == A.interpolate_linear(g0, g1, 0.4 + deltas[i]).xforms[1].e
        assert total == sum(counts) * iters == walkers * iters
