"""GPU: batched rendering (pyr3_batch_*): every genome of a batch agrees with
the same genome rendered alone through the per-genome path -- statistically,
since walker counts and seeds differ -- and gets exactly its samples.  Two
genomes of the batch share a structure, so each needs its own module
instance.  The last three genomes are large enough (>= 2^24 samples) to run
beside the graph through the per-genome path, one after another; two of
them share a structure with each other and with graph genomes (module
instance 0 beside the graph's instances)."""
import copy

import numpy as np
import pytest

from pyr3_b200 import batch as B
from pyr3_b200 import renderer as R
from pyr3_b200 import workloads

pytestmark = pytest.mark.gpu

W, H = 160, 120


def _genomes():
    a = workloads.plain_small()
    a2 = copy.deepcopy(a)  # same structure, other values
    rng = np.random.default_rng(8)
    for x in a2.xforms:
        x.a, x.b, x.c, x.d, x.e, x.f = (v + float(dv) for v, dv in
                                        zip((x.a, x.b, x.c, x.d, x.e, x.f), rng.uniform(-0.1, 0.1, 6)))
    b, _ = workloads.motion_4k()
    big = copy.deepcopy(a2)
    big2 = copy.deepcopy(b)
    big3 = copy.deepcopy(a)
    for x in big3.xforms:
        x.c, x.f = x.c + 0.05, x.f - 0.05
    gs = [a, a2, b, big, big2, big3]
    for g in gs:
        g.size = (W, H)
        g.oversample = 1
        g.density = None
        g.scale = W / 4
        g.quality = 640.0  # 1.2e7 samples each: in the graph
    for g in (big, big2, big3):
        g.quality = 3600.0  # 6.9e7 samples: beside the graph
    return gs


def _logd(h):
    return np.log1p(h.reshape(-1, 4)[:, 3].astype(np.float64) / 255.0)


def _single(g, seed):
    r = R.create_renderer(W, H, 1)
    walkers, iters, total = R.compute_dispatch(g.quality, W, H)
    r.reset(g)
    r.iterate(g, seed, walkers, iters)
    h, _, _ = r.read_histogram()
    s, _ = r.counters()
    r.destroy()
    return h, s


def test_batch_matches_per_genome_path():
    gs = _genomes()
    b = B.Batch(gs, n_streams=3, seed=5)
    b.run()
    ms, samples = b.sync()
    assert samples == sum(b.samples) and ms > 0
    for i, g in enumerate(gs):
        s, n_in = b.renderers[i].counters()
        assert s == b.samples[i]
        hb, _, _ = b.renderers[i].read_histogram()
        assert int(hb.reshape(-1, 4)[:, 3].astype(np.uint64).sum()) == 255 * n_in
        h1, _ = _single(g, 101)
        h2, _ = _single(g, 202)
        a, r1, r2 = _logd(hb), _logd(h1), _logd(h2)
        l1 = float(np.abs(a - r1).sum() / r1.sum())
        floor = float(np.abs(r2 - r1).sum() / r1.sum())
        print(f"genome {i}: batch vs single L1 {l1:.4%} (single-vs-single {floor:.4%})")
        assert l1 <= max(0.01, 1.5 * floor), (i, l1, floor)
    # a second run starts from cleared histograms
    b.run()
    b.sync()
    assert b.renderers[0].counters()[0] == b.samples[0]
    img = b.present(2)
    assert img.shape == (H, W, 4) and int(img[..., :3].max()) > 0
    b.destroy()
