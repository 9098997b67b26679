"""Batched rendering: many genomes of uneven structure and size in one CUDA
graph (pyr3_batch_* in the C-ABI).

Each genome gets its own renderer (histogram, palette, output) and its own
instance of its specialised chaos module; one graph launch clears every
histogram and runs every genome's chaos kernel, spread over worker streams
so that the launches run concurrently.  The walker count per genome is
chosen for the batch (see pyr3_batch_create); samples per genome follow
computeDispatch (src/renderer.ts:57-78) of its quality and canvas.

    b = Batch(workloads.batch_256())
    b.run(); ms, samples = b.sync()
    img = b.present(0)
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from .renderer import DEFAULT_WALKER_JITTER, GpuGenome, Renderer, compute_dispatch

GOLDEN = 0x9E3779B1


class Batch:
    def __init__(self, genomes, n_streams: int = 16, seed: int = 0, device: int = 0):
        self.genomes = list(genomes)
        n = len(self.genomes)
        self.renderers = []
        self.gpu = []
        self.samples = []
        opts = (_lib.IterateOpts * n)()
        gcs = (_lib.GenomeC * n)()
        hs = (C.c_void_p * n)()
        for i, g in enumerate(self.genomes):
            W, H = g.size
            r = Renderer(W, H, g.oversample or 1, g.filter_radius, device=device)
            r.reset(g)
            gg = GpuGenome(g)
            walkers, iters, total = compute_dispatch(g.quality or 16, W, H)
            self.renderers.append(r)
            self.gpu.append(gg)
            self.samples.append(total)
            o = opts[i]
            o.walkers, o.iters_per_walker = walkers, iters
            o.seed = (seed + i * GOLDEN) & 0xFFFFFFFF
            o.walker_jitter = DEFAULT_WALKER_JITTER
            o.flow_strength = o.trap_strength = o.phase_strength = o.phase_freq = 1.0
            gcs[i] = gg.c
            hs[i] = r.handle.value
        self._opts, self._gcs, self._hs = opts, gcs, hs
        self._b = C.c_void_p()
        _lib.check(_lib.lib().pyr3_batch_create(hs, gcs, opts, n, n_streams, C.byref(self._b)))

    def run(self) -> None:
        """Clear every histogram and accumulate every genome's samples."""
        _lib.check(_lib.lib().pyr3_batch_run(self._b))

    def sync(self):
        """Wait for the last run; (device ms, total samples)."""
        ms, s = C.c_float(), C.c_uint64()
        _lib.check(_lib.lib().pyr3_batch_sync(self._b, C.byref(ms), C.byref(s)))
        return ms.value, s.value

    def present(self, i: int, **kw):
        return self.renderers[i].present(self.genomes[i], self.samples[i], **kw)

    def destroy(self) -> None:
        if self._b:
            _lib.lib().pyr3_batch_destroy(self._b)
            self._b = C.c_void_p()
        for r in self.renderers:
            r.destroy()
        self.renderers = []

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
