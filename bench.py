"""pyr3-b200 benchmark: chaos-game iterations/s on one of the seeded
workloads (default: the headline 1080p, 12-xform + final configuration).

A step is one full frame of the hot path: reset (zero the histogram),
iterate (all quality x W x H post-fuse samples), present (density estimation
when the workload sets it, tonemap to RGBA8).  `value` is the device time of
the K timed steps (CUDA events on the renderer's stream, L2 flushed between
steps, inputs already resident); `e2e` is the same metric through the public
API with the palette / genome uploaded and the image read back every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl reference]

With --gpus N > 1 (launched by torchrun) every rank renders an independent
replica of the workload (the path has no exchange step: replicas only) and
rank 0 reports N x samples / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "headline": ("iters/s (1080p, 12 xforms)", "headline_1080p"),
    "plain_small": ("iters/s (640x480, 3 xforms)", "plain_small"),
    "motion_4k": ("iters/s (4K, 6 xforms, 8 temporal samples)", "motion_4k"),
    "batch_256": ("iters/s (256 genomes, batched)", "batch_256"),
    "denoise": ("denoiser training pixels/s (U-Net fwd+bwd+Adam)", "denoise_set"),
    "animate": ("iters/s (30 frames 640x360, 8 sub-frames each, batched)", "animate_preview"),
    "exposure": ("auto-exposure passes/s (1080p os 2 present + 1024-edge probe)", "headline_1080p"),
}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    def __init__(self, device: int):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={device}",
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap,utilization.gpu",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                util = float(f[6])
                if util < 50:
                    continue
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[2 + k].lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def _workload(name):
    """(genome, genome at shutter close or None)."""
    from pyr3_b200 import workloads

    g = getattr(workloads, CONFIGS[name][1])()
    if isinstance(g, tuple):  # motion blur: keyframes at shutter open and close
        return g
    if isinstance(g, list):  # batch: its first genome stands for it where one genome is needed
        return g[0], None
    return g, None


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        return ws, rank, local, dist
    return 1, 0, 0, None


def _max_over_ranks(x: float, dist, local: int) -> float:
    if dist is None:
        return x
    import torch

    dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


# --------------------------------------------------------------- CPU baseline
def cpu_reference_rate(g, target_seconds: float = 12.0, threads: int | None = None):
    """The reference's own chaos loop (its WGSL compiled for the CPU,
    oracle/_ref) on the host cores: a bounded sample of the workload
    (1024 walkers, the reference's TARGET_WALKERS, x fewer iterations)."""
    from oracle import oracle as O
    from pyr3_b200 import genome as G

    threads = threads or os.cpu_count() or 1
    ge = G.expand_for_gpu(g)
    xf = G.pack_xforms(ge)
    pal = G.bake_lut(ge.palette, ge.palette_hue, ge.palette_interp)
    w = np.array([x.weight for x in ge.xforms], np.float64)
    xa = G.xaos_matrix(ge)
    distrib = O.pack_xform_distrib(w, None if xa is None else xa.astype(np.float64))
    W, H = g.size
    os_ = g.oversample
    walkers = 1024

    def run(iters):
        u = np.zeros(31, np.uint32)
        f = u.view(np.float32)
        i32 = u.view(np.int32)
        u[0], u[1], u[2], u[3] = W * os_, H * os_, iters, 200
        f[4], f[5], f[6] = g.scale * os_, g.cx, g.cy
        u[7] = 1
        i32[8] = G.final_slot(ge)
        f[9] = np.float32(g.rotate * np.pi / 180.0)
        u[10] = 1 if g.palette_mode == "linear" else 0
        u[12] = walkers
        f[13] = 1e-7
        f[30] = g.xform_blend
        hist = np.zeros(W * os_ * H * os_ * 4, np.uint32)
        isaac = O.pack_isaac_states(walkers, 1)
        t0 = time.perf_counter()
        O.ref_chaos_run(u, xf, len(ge.xforms), pal, distrib, isaac, 0, walkers, hist, threads)
        return time.perf_counter() - t0

    probe_iters = 256
    dt = run(probe_iters)
    rate = walkers * (probe_iters + 200) / max(dt, 1e-6)
    iters = int(max(256, min(2_000_000, rate * target_seconds / walkers - 200)))
    dt = run(iters)
    samples = walkers * iters  # post-fuse samples
    return samples / dt, threads, f"{walkers} walkers x {iters} iterations (+200 fuse) of the workload genome"


def _config(args, g, g_close, samples, ws):
    """The workload description both arms print (identical for the same
    --config, so the two lines describe the same work)."""
    W, H = g.size
    return {"workload": args.config, "canvas": [W, H], "oversample": g.oversample,
            "quality_spp": g.quality, "samples_per_step": samples,
            "xforms": len(g.xforms), "final_xform": g.finalxform is not None,
            "density_estimation": g.density is not None,
            "temporal_samples": 8 if g_close is not None else 1,
            "l2": "256 MiB scratch overwritten between timed steps",
            "parallelism": f"replicas x{ws}"}


# ------------------------------------------------------------------ ours
def bench_ours(args, ws, rank, local, dist):
    from pyr3_b200 import _lib, renderer as R

    from pyr3_b200 import animate

    g, g_close = _workload(args.config)
    W, H = g.size
    os_ = g.oversample
    if args.samples:  # profiling case: same genome and canvas, fewer samples per step
        import copy

        g = copy.deepcopy(g)
        g.quality = args.samples / (W * H)
        if g_close is not None:
            g_close = copy.deepcopy(g_close)
            g_close.quality = g.quality
    walkers, iters, samples = R.compute_dispatch(g.quality, W, H)
    r = R.create_renderer(W, H, os_, g.filter_radius, device=local)
    gg = R.GpuGenome(g)
    r.prepare(gg)  # NVRTC specialisation (cached), outside the timed region
    lib = _lib.lib()
    h = r.handle
    p = r.present_opts(g)
    out_dev = None
    import torch  # device buffer for the present output

    out_dev = torch.empty((H, W, 4), dtype=torch.uint8, device=f"cuda:{local}")
    pal = None
    from pyr3_b200.genome import bake_lut

    pal = bake_lut(g.palette, g.palette_hue, g.palette_interp)
    L2_FLUSH = 256 << 20

    def step_device(seed):
        if g_close is None:
            _lib.check(lib.pyr3_reset(h, _lib.ptr(pal)))
            _lib.check(lib.pyr3_mark(h, 4))
            r.iterate(gg, seed, walkers, iters, kernel=args.kernel)
        else:  # one motion-blurred frame: 8 sub-frames into one histogram
            _lib.check(lib.pyr3_mark(h, 4))
            n, _ = animate.render_motion_frame(r, g, g_close, 0.5, ntemporal=8, seed=seed,
                                               kernel=args.kernel)
            assert n == samples
        _lib.check(lib.pyr3_mark(h, 5))
        _lib.check(lib.pyr3_present_device(h, C.byref(p), samples, C.c_void_p(out_dev.data_ptr()),
                                           _lib.OUT_RGBA8))

    for k in range(args.warmup):
        step_device(1000 + k)
    r.sync()
    _barrier(dist)
    clocks = Clocks(local) if rank == 0 else None
    total_ms, chaos_ms, present_ms = 0.0, [], []
    launches0 = r.launches
    for k in range(args.steps):
        _lib.check(lib.pyr3_flush_l2(h, L2_FLUSH))
        _lib.check(lib.pyr3_mark(h, 0))
        step_device(k)
        _lib.check(lib.pyr3_mark(h, 1))
        ms = C.c_float()
        _lib.check(lib.pyr3_elapsed(h, 0, 1, C.byref(ms)))
        total_ms += ms.value
        _lib.check(lib.pyr3_elapsed(h, 4, 5, C.byref(ms)))
        chaos_ms.append(ms.value)
        _lib.check(lib.pyr3_elapsed(h, 5, 1, C.byref(ms)))
        present_ms.append(ms.value)
    clk = clocks.stop() if clocks else None
    chaos_launches = r.launches - launches0
    n_samples, n_splats = r.counters()
    _barrier(dist)
    t_max = _max_over_ranks(total_ms, dist, local)

    # Scatter roofline: the same number of 4-atomic splats into uniformly
    # random cells of this histogram (pyr3_splat_rate), against the chaos
    # kernel's splats per second.  The histogram is reset by every step below.
    srate = None
    if n_splats > 0:
        sms = C.c_float()
        _lib.check(lib.pyr3_splat_rate(h, n_splats, C.byref(sms)))
        _lib.check(lib.pyr3_splat_rate(h, n_splats, C.byref(sms)))
        srate = n_splats / (sms.value / 1e3)

    # e2e through the public API: host palette + genome in, RGBA8 image out
    host_img = np.zeros((H, W, 4), np.uint8)
    def step_public(seed):
        if g_close is None:
            r.reset(g)
            r.iterate(g, seed, walkers, iters, kernel=args.kernel)
        else:
            animate.render_motion_frame(r, g, g_close, 0.5, ntemporal=8, seed=seed, kernel=args.kernel)
        r.present(g, samples, out=host_img)

    for k in range(max(1, args.warmup // 2)):
        step_public(5000 + k)
    e2e_ms, e2e_wall_ms = 0.0, 0.0
    for k in range(args.steps):
        _lib.check(lib.pyr3_flush_l2(h, L2_FLUSH))
        r.sync()
        t0 = time.perf_counter()
        _lib.check(lib.pyr3_mark(h, 2))
        step_public(7000 + k)  # ends with the blocking image read-back
        _lib.check(lib.pyr3_mark(h, 3))
        e2e_wall_ms += (time.perf_counter() - t0) * 1e3
        ms = C.c_float()
        _lib.check(lib.pyr3_elapsed(h, 2, 3, C.byref(ms)))
        e2e_ms += ms.value
    e2e_max = _max_over_ranks(e2e_wall_ms, dist, local)
    e2e_dev_max = _max_over_ranks(e2e_ms, dist, local)

    if rank != 0:
        r.destroy()
        return None
    value = ws * samples * args.steps / (t_max / 1e3)
    e2e = ws * samples * args.steps / (e2e_max / 1e3)
    e2e_dev = ws * samples * args.steps / (e2e_dev_max / 1e3)
    peak, peak_kind = _peaks()
    # Dominant kernel: the chaos kernel.  Algorithmic bytes: every in-canvas
    # splat reads and writes one 16-byte RGBA u32 bucket.  The counters
    # restart at every reset, so they hold the last timed step.  The wave
    # kernel advances every walker one iteration per launch, so a step is
    # many launches: bytes per launch / mean launch time = bytes per step /
    # chaos time per step (the time between the launches counted in).
    per_step_launches = max(1, chaos_launches // max(1, args.steps))
    splats_per_launch = n_splats / per_step_launches
    mean_chaos = statistics.mean(chaos_ms)
    achieved = n_splats * 32.0 / (mean_chaos / 1e3) / 1e9
    traffic = None  # DRAM bytes per launch measured by ncu for this workload at full size
    tpath = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "roofline_traffic.json")
    if not args.samples and os.path.exists(tpath):
        t = json.load(open(tpath)).get(args.config)
        traffic = t["dram_bytes_per_launch"] if t else None
    h2d = 4096 + gg.xforms.nbytes + (len(g.xforms) + 1) * len(g.xforms) * 2
    line = {
        "metric": CONFIGS[args.config][0], "value": value, "unit": "iters/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded genome, pyr3_b200/workloads.py)",
        "config": _config(args, g, g_close, samples, ws),
        "chaos_kernel": args.kernel,
        "e2e": {"value": e2e, "unit": "iters/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(host_img.nbytes),
                "device_value": e2e_dev,
                "note": "host wall clock around each public-API step (palette and genome upload, "
                        "iterate, present, RGBA8 read back to host memory); device_value = the same "
                        "steps timed by CUDA events on the renderer's stream"}, 
        "chaos_kernel_ms": mean_chaos,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "note": f"chaos kernel, {per_step_launches} launches per step; algorithmic bytes = "
                             f"32 B (16 B bucket read+write) per in-canvas splat ({splats_per_launch:.0f} "
                             f"splats per launch); peak {peak_kind}; the kernel is bound by instruction "
                             f"issue and latency (ncu), not by HBM"},
        "scatter_roofline": None if srate is None else {
            "achieved": n_splats / (mean_chaos / 1e3), "peak": srate, "unit": "splats/s",
            "frac": n_splats / (mean_chaos / 1e3) / srate,
            "note": "a splat = 4 saturating u32 atomics on one 16-byte bucket; peak = the same splats "
                    "into uniformly random buckets of this histogram (pyr3_splat_rate), measured here"},
        "present_roofline": _present_roofline(g, present_ms, peak, peak_kind),
        "gpu_launches": chaos_launches + args.steps * (1 + (1 if g.density is not None else 0)),
        "clocks": clk,
    }
    if ws == 1 and not args.no_cpu_baseline:
        rate, cores, sample = cpu_reference_rate(g)
        line["cpu_baseline"] = {"value": rate, "unit": "iters/s", "cores": cores, "kind": "reference",
                                "sample": sample}
    r.destroy()
    return line


def _present_roofline(g, present_ms, peak, peak_kind):
    """HBM roofline of the present (density estimation when the workload
    sets it, then tonemap to RGBA8), from its CUDA-event time per step.
    Algorithmic bytes: the histogram read once (16 B per super-sampled
    bucket) and the image written (4 B per pixel); with density estimation
    also the filtered buckets written and read once more (2 x 16 B)."""
    W, H = g.size
    n_super = W * H * g.oversample * g.oversample
    nbytes = n_super * 16 + W * H * 4 + (2 * n_super * 16 if g.density is not None else 0)
    ms = statistics.mean(present_ms)
    achieved = nbytes / (ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "ms": ms, "bytes": nbytes,
            "note": ("density estimation + tonemap" if g.density is not None else "tonemap") +
                    f"; the disc spreading of density estimation is bound by shared-memory accumulation, "
                    f"not HBM; peak {peak_kind}"}


def bench_batch(args, ws, rank, local, dist):
    """A step = one graph launch rendering all 256 genomes (each histogram
    cleared, every genome's samples accumulated)."""
    from pyr3_b200 import batch as B
    from pyr3_b200 import workloads

    gs = workloads.batch_256()
    b = B.Batch(gs, n_streams=16, seed=11, device=local)
    for _ in range(args.warmup):
        b.run()
    b.sync()
    _barrier(dist)
    clocks = Clocks(local) if rank == 0 else None
    total_ms = 0.0
    launches = 0
    for _ in range(args.steps):
        _lib_flush(b)
        b.run()
        ms, samples = b.sync()
        total_ms += ms
        # graph genomes: one chaos kernel each; the others ran through
        # pyr3_iterate, which counts its own launches
        launches += sum(1 if s < (1 << 24) else r.last_iterate_launches()
                        for s, r in zip(b.samples, b.renderers))
    clk = clocks.stop() if clocks else None
    t_max = _max_over_ranks(total_ms, dist, local)
    # e2e through the public API: every genome's image read back to the host
    import time as _t

    d2h = sum(g.size[0] * g.size[1] * 4 for g in gs)
    e2e_ms = 0.0
    for _ in range(args.steps):
        t0 = _t.perf_counter()
        b.run()
        b.sync()
        for i in range(len(gs)):
            b.present(i)
        e2e_ms += (_t.perf_counter() - t0) * 1e3
    e2e_max = _max_over_ranks(e2e_ms, dist, local)
    # The same genomes one after another through the per-genome path
    # (pyr3_iterate, autotuned kernel), device time; the first pass loads
    # the modules and runs the autotuner, the second is the one reported.
    from pyr3_b200.renderer import compute_dispatch

    seq_ms = 0.0
    for _ in range(2):
        seq_ms = 0.0
        for i, g in enumerate(gs):
            r = b.renderers[i]
            w, it, _n = compute_dispatch(g.quality or 16, *g.size)
            r.reset(g)
            r.iterate(b.gpu[i], seed=11 + i, walkers=w, iters_per_walker=it)
            seq_ms += r.last_iterate_ms()
    seq_max = _max_over_ranks(seq_ms, dist, local)
    b.destroy()
    if rank != 0:
        return None
    value = ws * samples * args.steps / (t_max / 1e3)
    peak, peak_kind = _peaks()
    return {
        "metric": CONFIGS[args.config][0], "value": value, "unit": "iters/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (256 seeded genomes, pyr3_b200/workloads.py)",
        "config": {"workload": args.config, "genomes": len(gs), "samples_per_step": samples,
                   "xforms": "2-20", "canvases": "256^2 / 512^2 / 800x600 / 1024x768",
                   "quality_spp": "50-400", "streams": 16,
                   "l2": "256 MiB scratch overwritten between timed steps",
                   "parallelism": f"replicas x{ws}"},
        "e2e": {"value": ws * samples * args.steps / (e2e_max / 1e3), "unit": "iters/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(d2h),
                "note": "graph launch + per-genome tonemap and RGBA8 readback; genomes uploaded once"},
        "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                     "traffic": None, "note": f"chaos kernels bound by issue/latency; peak {peak_kind}"},
        "per_genome_path": {"value": ws * samples / (seq_max / 1e3), "unit": "iters/s",
                            "note": "the same genomes one after another through pyr3_iterate "
                                    "(autotuned kernel), device time"},
        "gpu_launches": launches,
        "clocks": clk,
    }


def _lib_flush(b):
    from pyr3_b200 import _lib

    _lib.check(_lib.lib().pyr3_flush_l2(b.renderers[0].handle, 256 << 20))
    b.renderers[0].sync()  # the flush runs on renderer 0's stream: finish it before the graph


def bench_reference(args, ws, rank, local, dist):
    """The reference's own chaos loop on the host cores, on the workload our
    arm runs: each step is a bounded sample of that workload (1024 walkers,
    fewer iterations), timed on the host clock; value = post-fuse samples
    per second of the timed steps."""
    if rank != 0:
        return None
    from pyr3_b200 import renderer as R

    g, g_close = _workload(args.config)
    _, _, samples = R.compute_dispatch(g.quality, *g.size)
    per = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_reference_rate(g, target_seconds=per)
    rates, times = [], []
    sample = ""
    cores = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rate, cores, sample = cpu_reference_rate(g, target_seconds=per)
        times.append(time.perf_counter() - t0)
        rates.append(rate)
    value = statistics.mean(rates)
    return {"impl": "reference", "metric": CONFIGS[args.config][0], "value": value, "unit": "iters/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded genome, pyr3_b200/workloads.py)",
            "config": (_config(args, g, g_close, samples, ws) if args.config not in ("batch_256", "animate")
                       else {"workload": args.config, "note": "the reference timed on the workload's "
                                                              "first genome"}),
            "cpu_baseline": {"value": value, "unit": "iters/s", "cores": cores, "kind": "reference",
                             "sample": f"per step {sample}, extrapolated per post-fuse sample; the "
                                       f"reference's chaos_main (src/shaders/chaos.wgsl) compiled "
                                       f"for the CPU"},
            "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def bench_denoise(args, ws, rank, local, dist):
    """Learned denoiser: a step = 200 Adam steps on batches of --dn-batch
    random --dn-crop square crops (default 32 x 256^2) from the training
    genomes' renders (25 spp features, 2000 spp target; --dn-genomes
    genomes at --dn-size, default 136 at 384^2, the last 8 held out);
    afterwards the held-out genomes are denoised and scored (PSNR and SSIM
    against their 2000-spp renders, and the plain spp that matches)."""
    import time as _t

    import torch

    from pyr3_b200 import denoise as DN
    from pyr3_b200 import workloads

    n_gen, size, n_ho = args.dn_genomes, args.dn_size, args.dn_held_out
    gs = workloads.denoise_set(seed=5 + 1000 * rank, n=n_gen, size=size)
    t0 = _t.perf_counter()
    xs, ts = DN.make_dataset(gs)
    render_s = _t.perf_counter() - t0
    n_tr = n_gen - n_ho
    xtr, ttr, xho, tho = xs[:n_tr], ts[:n_tr], xs[n_tr:], ts[n_tr:]
    per = 200
    batch, crop = args.dn_batch, args.dn_crop
    in_ch = args.dn_input
    net, _, _ = DN.train(xtr, ttr, steps=per * args.warmup, batch=batch, crop=crop, seed=1, in_ch=in_ch)
    params = net.params()
    torch.cuda.synchronize()
    _barrier(dist)
    clocks = Clocks(local) if rank == 0 else None
    net, losses, ms = DN.train(xtr, ttr, steps=per * args.steps, batch=batch, crop=crop, seed=2,
                               params=params, in_ch=in_ch, lr_end=args.dn_lr_end)
    launches = net.launches
    clk = clocks.stop() if clocks else None
    t_max = _max_over_ranks(ms, dist, local)
    p_noisy, p_dn, dn_img = DN.evaluate(net.params(), xho, tho, in_ch=in_ch)
    ssim_in = DN.ssim(np.clip(xho[:, DN.IN_CH:DN.IN_CH + DN.OUT_CH], 0.0, 1.0), tho)
    ssim_dn = DN.ssim(dn_img, tho)
    # time to quality: plain renders of the held-out genomes at rising spp against the
    # same 2000-spp targets, and the denoiser's inference time for all of them
    plain = DN.plain_quality(gs[n_tr:], tho, (25, 50, 100, 200, 400, 800))
    inet = DN.UNet(len(xho), size, size, net.params(), in_ch=in_ch)
    inet.set_batch(xho)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    inet.forward()
    e0.record()
    inet.forward()
    e1.record()
    e1.synchronize()
    infer_ms = e0.elapsed_time(e1)
    match = next((p for p in plain if p[1] >= p_dn), None)
    # e2e: batches assembled on the host, uploaded each step, loss read back each step
    rng = np.random.default_rng(3)
    hnet = DN.UNet(batch, crop, crop, net.params(), in_ch=in_ch)
    hnet.capture()
    n_e2e = max(20, per * 8 * 128 * 128 // (batch * crop * crop))  # host-assembled batches: ~200 of 8 x 128^2
    hx = np.empty((batch, DN.IN_CH + DN.OUT_CH, crop, crop), np.float32)
    ht = np.empty((batch, 3, crop, crop), np.float32)
    torch.cuda.synchronize()
    t0 = _t.perf_counter()
    for _ in range(n_e2e):
        idx = rng.integers(0, n_tr, batch)
        yy, xx = rng.integers(0, size - crop + 1, batch), rng.integers(0, size - crop + 1, batch)
        for j in range(batch):
            hx[j] = xtr[idx[j], :, yy[j]:yy[j] + crop, xx[j]:xx[j] + crop]
            ht[j] = ttr[idx[j], :, yy[j]:yy[j] + crop, xx[j]:xx[j] + crop]
        hnet.set_batch(hx, ht)
        hnet.replay()
        hnet.step()
        hnet.read_loss()
    e2e_s = _t.perf_counter() - t0
    e2e_max = _max_over_ranks(e2e_s * 1e3, dist, local)
    if rank != 0:
        return None
    pix_step = batch * crop * crop
    value = ws * pix_step * per * args.steps / (t_max / 1e3)
    flop_pix = 3.0 * DN.flops_per_pixel(in_ch=in_ch)  # forward + data and weight gradients
    achieved = value / ws * flop_pix / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, pk = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        peak, pk = 1590.0, "fallback"
    return {
        "metric": CONFIGS["denoise"][0], "value": value, "unit": "pixels/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic ({n_gen} seeded genomes, pyr3_b200/workloads.py:denoise_set, rendered here)",
        "config": {"workload": "denoise", "unet_levels": len(DN.CHANS), "channels": list(DN.CHANS),
                   "params": DN.param_count(in_ch=in_ch), "canvas": [size, size], "spp_input": 25, "spp_target": 2000,
                   "input_channels": in_ch, "train_genomes": n_tr, "held_out_genomes": n_ho,
                   "batch": batch, "crop": crop,
                   "adam_steps_per_step": per, "lr": [1e-3, args.dn_lr_end if args.dn_lr_end is not None else 1e-3],
                   "l2": "inputs resident; working set < L2 per layer",
                   "parallelism": f"replicas x{ws}"},
        "quality": {"held_out_psnr_input_db": p_noisy, "held_out_psnr_denoised_db": p_dn,
                    "held_out_ssim_input": ssim_in, "held_out_ssim_denoised": ssim_dn,
                    "plain_render_psnr_by_spp": [[p[0], round(p[1], 3), round(p[2], 3)] for p in plain],
                    "plain_spp_matching_denoised": match[0] if match else None,
                    "time_to_denoised_quality_ms": {"denoised": round(plain[0][2] + infer_ms, 3),
                                                    "plain": round(match[2], 3) if match else None},
                    "train_loss_first_last": [losses[0][1], losses[-1][1]],
                    "adam_steps_total": per * (args.warmup + args.steps), "render_seconds": render_s},
        "e2e": {"value": ws * pix_step * n_e2e / (e2e_max / 1e3), "unit": "pixels/s",
                "h2d_bytes_per_step": int(hx.nbytes + ht.nbytes) * per, "d2h_bytes_per_step": 4 * per},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "note": f"FLOPs = 3 x 2 x sum(ci co 9 H_l W_l) per pixel = {flop_pix:.0f}; forward and "
                             f"data-gradient convolutions and the weight gradients on tcgen05 (bf16 operands, f32 "
                             f"accumulation); staging f32 NCHW tensors into bf16 operands bounds them; peak = bf16 "
                             f"dense, {pk}"},
        "gpu_launches": launches,
        "clocks": clk,
    }


def bench_animate(args, ws, rank, local, dist):
    """Animation frames (bin/pyr3-animate.ts frame loop, src/animate-render.ts
    renderAnimationFrame): a step = 30 frames (1 s at 30 fps) of the moving
    6-xform genome at 640x360, 50 spp, 8 box-filtered sub-frames each -- 240
    sub-frame genomes in one AnimationBatch graph launch -- then every frame
    presented (DE + tonemap) into a device buffer.  The step spans the
    batch's streams and the 30 renderers' streams, so it is timed on the
    host clock between device synchronisations."""
    import time as _t

    import torch

    from pyr3_b200 import animate as A
    from pyr3_b200 import workloads

    g0, g1 = workloads.animate_preview()
    W, H = g0.size
    times = [k / 30 for k in range(30)]
    ab = A.AnimationBatch(g0, g1, times, ntemporal=8, seed=7, device=local)
    outs = [torch.empty((H, W, 4), dtype=torch.uint8, device=f"cuda:{local}") for _ in times]
    torch.cuda.synchronize()

    def step(to_host=False):
        ab.run()
        ab.sync()
        for k in range(len(times)):
            if to_host:
                ab.present(k)
            else:
                ab.renderers[k].present_device(ab.centres[k], ab.samples[k], outs[k].data_ptr())
        for r in ab.renderers:
            r.sync()

    for _ in range(args.warmup):
        step()
    _barrier(dist)
    clocks = Clocks(local) if rank == 0 else None
    graph_ms = 0.0
    t0 = _t.perf_counter()
    for _ in range(args.steps):
        step()
        graph_ms += ab.sync()[0]
    step_s = (_t.perf_counter() - t0) / args.steps
    clk = clocks.stop() if clocks else None
    t0 = _t.perf_counter()
    for _ in range(args.steps):
        step(to_host=True)
    e2e_s = (_t.perf_counter() - t0) / args.steps
    # The reference's shape: one frame after another through
    # render_motion_frame on one renderer (pyr3_iterate per sub-frame), each
    # presented; the first pass loads modules, the second is reported.
    from pyr3_b200 import renderer as R

    r1 = R.create_renderer(W, H, 1, device=local)
    seq_s = 0.0
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = _t.perf_counter()
        for k, t in enumerate(times):
            n, _ = A.render_motion_frame(r1, g0, g1, t, ntemporal=8, seed=7)
            r1.present_device(ab.centres[k], n, outs[k].data_ptr())
        r1.sync()
        seq_s = _t.perf_counter() - t0
    r1.destroy()
    samples = sum(ab.samples)
    t_max = _max_over_ranks(step_s * 1e3, dist, local)
    e2e_max = _max_over_ranks(e2e_s * 1e3, dist, local)
    seq_max = _max_over_ranks(seq_s * 1e3, dist, local)
    n_gen = ab.n_genomes
    ab.destroy()
    if rank != 0:
        return None
    peak, peak_kind = _peaks()
    return {
        "metric": CONFIGS["animate"][0], "value": ws * samples / (t_max / 1e3), "unit": "iters/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (motion_4k keyframes at 640x360, pyr3_b200/workloads.py:animate_preview)",
        "config": {"workload": "animate", "frames": len(times), "fps": 30, "canvas": [W, H],
                   "quality_spp": g0.quality, "ntemporal": 8, "sub_frame_genomes": n_gen,
                   "samples_per_step": samples, "frames_per_s": ws * len(times) / (t_max / 1e3),
                   "graph_ms_per_step": graph_ms / args.steps,
                   "timing": "host clock between synchronisations (batch + 30 renderer streams)",
                   "l2": "30 histograms of 3.7 MB (110 MB) rewritten every step",
                   "parallelism": f"replicas x{ws}"},
        "e2e": {"value": ws * samples / (e2e_max / 1e3), "unit": "iters/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": W * H * 4 * len(times),
                "note": "every frame's RGBA8 image read back to the host"},
        "per_frame_path": {"value": ws * samples / (seq_max / 1e3), "unit": "iters/s",
                           "frames_per_s": ws * len(times) / (seq_max / 1e3),
                           "note": "the same frames one after another (render_motion_frame: one "
                                   "pyr3_iterate per sub-frame, then present), host clock"},
        "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                     "traffic": None, "note": f"chaos kernels bound by issue/latency; peak {peak_kind}"},
        "gpu_launches": (n_gen + 2 * len(times)) * args.steps,
        "clocks": clk,
    }


def bench_exposure(args, ws, rank, local, dist):
    """Render-time auto-exposure (bin/pyr3-render.ts:487-513) after the
    headline render: a step = the preview probe (1024 x 576, 16 spp, fixed
    seed: chaos, present, device mean luminance) and the brightness fit on
    the 1920x1080 os-2 histogram (present, device mean, up to 4
    re-presents; 8 bytes read back per pass).  The loop is host-driven, so
    a step is timed on the host clock between device synchronisations."""
    import time as _t

    import torch

    from oracle import auto_exposure as OA
    from oracle import oracle as O
    from pyr3_b200 import _lib, auto_exposure as AE, renderer as R

    g, _ = _workload("headline")
    W, H = g.size
    r = R.create_renderer(W, H, g.oversample, g.filter_radius, device=local)
    walkers, iters, samples = R.compute_dispatch(g.quality, W, H)
    if args.samples:  # profiling case: a smaller high-quality histogram (untimed)
        walkers, iters = 1024, max(1, args.samples // 1024)
        samples = walkers * iters
    r.reset(g)
    r.iterate(g, 1, walkers, iters)
    probe_r = R.create_renderer(16, 16, 1, device=local)
    img = torch.empty((H, W, 4), dtype=torch.uint8, device=f"cuda:{local}")
    host = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True)
    lib = _lib.lib()

    def step(e2e=False):
        target = AE.measure_probe_luminance(g, renderer=probe_r)
        fit, _ = AE.auto_expose(r, g, samples, target, image=img)
        if e2e:
            host.copy_(img)
        return target, fit

    per = 20  # passes per bench step, so the clock sampler sees the timed region
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    _barrier(dist)
    clocks = Clocks(local) if rank == 0 else None
    l0 = r.launches + probe_r.launches
    t0 = _t.perf_counter()
    for _ in range(args.steps * per):
        target, fit = step()
    torch.cuda.synchronize()
    step_s = (_t.perf_counter() - t0) / (args.steps * per)
    chaos_launches = (r.launches + probe_r.launches - l0) / (args.steps * per)
    clk = clocks.stop() if clocks else None
    t0 = _t.perf_counter()
    for _ in range(args.steps * per):
        step(e2e=True)
    torch.cuda.synchronize()
    e2e_s = (_t.perf_counter() - t0) / (args.steps * per)
    # the luminance pass alone: device time of pyr3_mean_luminance on the
    # 1080p image (memset, kernel, 8-byte read-back)
    out = C.c_double()
    reps = 50
    _lib.check(lib.pyr3_mark(r.handle, 2))
    for _ in range(reps):
        _lib.check(lib.pyr3_mean_luminance(r.handle, C.c_void_p(img.data_ptr()), W * H, _lib.OUT_RGBA8,
                                           C.byref(out)))
    _lib.check(lib.pyr3_mark(r.handle, 3))
    lms = C.c_float()
    _lib.check(lib.pyr3_elapsed(r.handle, 2, 3, C.byref(lms)))
    luma_ms = lms.value / reps
    t_max = _max_over_ranks(step_s * 1e3, dist, local)
    e2e_max = _max_over_ranks(e2e_s * 1e3, dist, local)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # one re-present pass the reference's way: its visualize shader on
        # the host cores over the super-res histogram, then the host mean
        hist, _, _ = r.read_histogram()
        p = r.present_opts(g)
        k1, k2 = O.derive_calibration(g.scale, samples, p.brightness, g.oversample)
        threads = os.cpu_count() or 1
        t0 = _t.perf_counter()
        ref = O.ref_visualize(W, H, g.oversample, O.spatial_kernel(0.5, g.oversample), np.float32(k1),
                              np.float32(k2), p.gamma, p.vibrancy, p.highpow, p.linrange,
                              bg=tuple(p.background), src_u32=hist.reshape(-1), threads=threads)
        OA.mean_luminance(np.clip(np.rint(ref * 255.0), 0, 255).astype(np.uint8))
        cpu_s = _t.perf_counter() - t0
        cpu = {"value": 1.0 / cpu_s, "unit": "re-present passes/s", "cores": threads, "kind": "reference",
               "sample": "one 1920x1080 os-2 visualize (the reference's shader on the CPU) + host mean "
                         "luminance; a full auto-exposure pass adds the probe render and 1-4 more presents"}
    if rank != 0:
        return None
    peak, pk = _peaks()
    luma_gbs = W * H * 4 / (luma_ms * 1e-3) / 1e9
    return {
        "metric": CONFIGS["exposure"][0], "value": ws * 1e3 / t_max, "unit": "passes/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max * per,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (headline genome, pyr3_b200/workloads.py:headline_1080p)",
        "config": {"workload": "exposure", "canvas": [W, H], "oversample": g.oversample,
                   "hq_samples": samples, "probe": [1024, 576], "probe_spp": 16,
                   "passes_per_step": per, "ms_per_pass": t_max,
                   "probe_target_mean": target, "fit": vars(fit),
                   "timing": "host clock between synchronisations (host-driven loop)",
                   "l2": "histogram 133 MB > L2", "parallelism": f"replicas x{ws}"},
        "e2e": {"value": ws * 1e3 / e2e_max, "unit": "passes/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(W * H * 4 + 8 * (2 + fit.iters)) * per},
        "roofline": {"bound": "hbm", "achieved": luma_gbs, "peak": peak, "unit": "GB/s",
                     "frac": luma_gbs / peak, "traffic": None,
                     "note": f"luminance pass: {W * H * 4} B image read per call / device time of "
                             f"pyr3_mean_luminance ({luma_ms * 1e3:.1f} us incl. memset and 8-byte read-back); "
                             f"the pass's dominant kernel is the probe's chaos kernel (9.4e6 samples, 200 "
                             f"burn-in iterations per walker), reported by the headline config; peak {pk}"},
        "cpu_baseline": cpu,
        "gpu_launches": int((chaos_launches + 2 * (1 + fit.iters) + 2) * per),
        "clocks": clk,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="headline", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel", default="auto", choices=["auto", "barrier", "queue", "wave"],
                    help="chaos kernel (auto: the autotuner's choice)")
    ap.add_argument("--dn-genomes", type=int, default=136,
                    help="denoise: seeded genomes rendered for the dataset (the last --dn-held-out held out)")
    ap.add_argument("--dn-size", type=int, default=384, help="denoise: canvas side of the dataset renders")
    ap.add_argument("--dn-held-out", type=int, default=8, help="denoise: genomes held out for scoring")
    ap.add_argument("--dn-batch", type=int, default=32, help="denoise: crops per Adam step")
    ap.add_argument("--dn-lr-end", type=float, default=None,
                    help="denoise: learning rate the timed steps fall to linearly (from 1e-3)")
    ap.add_argument("--dn-crop", type=int, default=256, help="denoise: crop side (a multiple of 16)")
    ap.add_argument("--dn-input", type=int, default=8, choices=[8, 11],
                    help="denoise: network input channels: the 8 features, or 11 with the noisy RGB")
    ap.add_argument("--samples", type=int, default=0,
                    help="override samples per step (small profiling case; not a bench number)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    ws, rank, local, dist = _dist()
    try:
        if args.impl == "reference" and args.config == "denoise":
            line = {"impl": "reference", "unavailable": "the reference has no learned denoiser"} \
                if rank == 0 else None
        elif args.impl == "reference" and args.config == "exposure":
            line = {"impl": "reference", "unavailable": "the reference presents only through WebGPU "
                    "(unavailable on this box); its visualize shader on the CPU is the cpu_baseline"} \
                if rank == 0 else None
        elif args.impl == "reference":
            line = bench_reference(args, ws, rank, local, dist)
        elif args.config == "batch_256":
            line = bench_batch(args, ws, rank, local, dist)
        elif args.config == "denoise":
            line = bench_denoise(args, ws, rank, local, dist)
        elif args.config == "exposure":
            line = bench_exposure(args, ws, rank, local, dist)
        elif args.config == "animate":
            line = bench_animate(args, ws, rank, local, dist)
        else:
            line = bench_ours(args, ws, rank, local, dist)
        if line is not None:
            print(json.dumps(line))
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
