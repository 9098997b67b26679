"""Learned denoiser: a small U-Net that maps a low-sample render (8 feature
channels) to the colours of a high-sample render of the same genome,
trained and run with this library's CUDA layers (pyr3_dn_* in the C-ABI):
the convolutions and their weight gradients on the tensor cores (tcgen05,
bf16 operands, f32 accumulation) by default, or all in f32.
The denoiser has no counterpart in the reference.

PyTorch only allocates device memory and supplies the stream here; every
layer, gradient and optimiser step is a kernel of libpyr3cuda.so, and the
module fails loudly without a GPU.

Architecture (chans = (16, 24, 32, 40, 48), ~195 k parameters): encoder
level l = two 3x3 conv + ReLU (input: the features, or the 2x2 average pool
of level l-1); decoder level l = nearest 2x upsample of the level below
concatenated with the encoder's level-l output, two 3x3 conv + ReLU; a last
3x3 conv to 3 channels added to the noisy image (the input's last three
channels, after the features).
Parameters are one flat f32 vector: per conv, weight [co][ci][3][3] then
bias[co].  Each encoder output is written straight into its decoder level's
concatenation buffer, so the skip connection costs no copy.

Input of a render (features()): 8 feature channels -- log density
log1p(hits), the normalised RGB accumulators (colour sums / count, 3),
alpha, the hit count per sample per pixel, the local 3x3 variance of the
noisy image's luminance, and the density-estimation radius the adaptive
filter would give the pixel (max_rad / (hits + 1)^curve, clamped, over
max_rad) -- then the noisy tonemapped RGB (3) as the residual's base.  Hits
are the pixel's bucket counts / 255 summed over its oversample block.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

CHANS = (16, 24, 32, 40, 48)
IN_CH, OUT_CH = 8, 3  # feature channels, output (and noisy-image) channels
IN_CH_WITH_RGB = IN_CH + OUT_CH  # a network may also read the noisy image as input


def layer_shapes(chans=CHANS, in_ch=IN_CH, out_ch=OUT_CH):
    """(co, ci) of every conv in parameter order."""
    L = len(chans)
    shapes = []
    for l in range(L):
        shapes += [(chans[l], in_ch if l == 0 else chans[l - 1]), (chans[l], chans[l])]
    for l in range(L - 2, -1, -1):
        shapes += [(chans[l], chans[l + 1] + chans[l]), (chans[l], chans[l])]
    shapes.append((out_ch, chans[0]))
    return shapes


def param_count(chans=CHANS, in_ch=IN_CH):
    return sum(co * ci * 9 + co for co, ci in layer_shapes(chans, in_ch))


def flops_per_pixel(chans=CHANS, in_ch=IN_CH):
    """Multiply-adds x 2 of one forward pass per full-resolution pixel."""
    f = 0.0
    L = len(chans)
    shapes = layer_shapes(chans, in_ch)
    for i, (co, ci) in enumerate(shapes):
        if i < 2 * L:
            lvl = i // 2
        elif i < len(shapes) - 1:
            lvl = L - 2 - (i - 2 * L) // 2
        else:
            lvl = 0
        f += 2.0 * co * ci * 9 / (4 ** lvl)
    return f


def _check(rc):
    _lib.check(rc)


class UNet:
    """Device-resident U-Net for images of N x (IN_CH + OUT_CH) x H x W (H, W
    multiples of 2^(levels-1)): the first convolution reads channels
    0..in_ch-1 (the features, and with in_ch = IN_CH_WITH_RGB also the noisy
    image), and the output is added to channels IN_CH..IN_CH+2.  forward() then backward() computes the parameter
    gradient of the MSE against a target; step() applies Adam."""

    def __init__(self, n: int, h: int, w: int, params: np.ndarray, chans=CHANS, device: int = 0,
                 tensor_cores: bool = True, in_ch: int = IN_CH):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("pyr3_b200.denoise needs a CUDA device")
        L = len(chans)
        if h % (1 << (L - 1)) or w % (1 << (L - 1)):
            raise ValueError(f"H and W must be multiples of {1 << (L - 1)}")
        self.t = torch
        self.tc = tensor_cores  # forward and data-gradient convolutions on tcgen05 (bf16 operands)
        self.dev = torch.device("cuda", device)
        self.n, self.h, self.w, self.chans = n, h, w, tuple(chans)
        self.L = L
        if in_ch not in (IN_CH, IN_CH_WITH_RGB):
            raise ValueError(f"in_ch must be {IN_CH} or {IN_CH_WITH_RGB}")
        self.in_ch = in_ch  # input channels the first convolution reads, from channel 0
        self.shapes = layer_shapes(chans, in_ch)
        self.offs = []
        o = 0
        for co, ci in self.shapes:
            self.offs.append((o, o + co * ci * 9))
            o += co * ci * 9 + co
        if params.size != o:
            raise ValueError(f"expected {o} parameters, got {params.size}")
        f32 = dict(dtype=torch.float32, device=self.dev)
        self.p = torch.tensor(params.astype(np.float32), **f32)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.steps = 0
        self.launches = 0  # kernels this network has queued
        self.wt = torch.zeros(max(co * ci * 9 for co, ci in self.shapes), **f32)  # flipped weights
        lib = _lib.lib()
        self.wsc_n = max(lib.pyr3_dn_wgrad_scratch_floats(co, ci) for co, ci in self.shapes)
        self.wsc = torch.zeros(self.wsc_n, **f32)  # weight-gradient partials
        hs = [(h >> l, w >> l) for l in range(L)]
        self.hs = hs
        z = lambda c, l: torch.zeros((n, c, hs[l][0], hs[l][1]), **f32)  # noqa: E731
        self.x = z(IN_CH + OUT_CH, 0)  # features, then the noisy image the output is added to
        self.tgt = z(OUT_CH, 0)
        self.out = z(OUT_CH, 0)
        self.gout = z(OUT_CH, 0)
        self.loss = torch.zeros(1, **f32)
        # encoder: a_l, inp_l (pooled input, l > 0); e_l lives in cat_l (l < L-1) or bottom
        self.a = [z(chans[l], l) for l in range(L)]
        self.inp = [self.x] + [z(chans[l - 1], l) for l in range(1, L)]
        self.cat = [z(chans[l + 1] + chans[l], l) for l in range(L - 1)]
        self.bottom = z(chans[L - 1], L - 1)
        self.da = [z(chans[l], l) for l in range(L - 1)]
        self.d = [z(chans[l], l) for l in range(L - 1)]
        # gradients
        self.gcat = [z(chans[l + 1] + chans[l], l) for l in range(L - 1)]
        self.gbottom = z(chans[L - 1], L - 1)
        self.gd = [z(chans[l], l) for l in range(L - 1)]
        self.gtmp = [z(max(chans[l], chans[l - 1] if l else 1), l) for l in range(L)]
        self.ginp = [None] + [z(chans[l - 1], l) for l in range(1, L)]

    # ---- tensor views: (pointer, per-image stride)
    @staticmethod
    def _v(t, c0=0):
        hw = t.shape[2] * t.shape[3]
        return C.c_void_p(t.data_ptr() + 4 * c0 * hw), t.shape[1] * hw

    def _e(self, l):
        """Encoder level l's output view (inside cat_l, after the upsampled channels)."""
        if l == self.L - 1:
            return self._v(self.bottom)
        return self._v(self.cat[l], self.chans[l + 1])

    def _ge(self, l):
        if l == self.L - 1:
            return self._v(self.gbottom)
        return self._v(self.gcat[l], self.chans[l + 1])

    def _w(self, i):
        a, b = self.offs[i]
        return C.c_void_p(self.p.data_ptr() + 4 * a), C.c_void_p(self.p.data_ptr() + 4 * b)

    def _gw(self, i):
        a, b = self.offs[i]
        return C.c_void_p(self.g.data_ptr() + 4 * a), C.c_void_p(self.g.data_ptr() + 4 * b)

    def _stream(self):
        return C.c_void_p(self.t.cuda.current_stream(self.dev).cuda_stream)

    def _conv(self, src, ci, dst, co, l, i, relu, bias=True):
        self.launches += 1
        w, b = self._w(i)
        h, wd = self.hs[l]
        fn = _lib.lib().pyr3_dn_conv3x3_bf16 if self.tc else _lib.lib().pyr3_dn_conv3x3
        _check(fn(src[0], src[1], ci, dst[0], dst[1], co, self.n, h, wd, w, b if bias else None,
                  1 if relu else 0, self._stream()))

    def _dgrad(self, g, co, dst, ci, l, i):
        """dst = input gradient of conv i (co <- ci) from its output gradient g."""
        self.launches += 2
        w, _ = self._w(i)
        L_ = _lib.lib()
        _check(L_.pyr3_dn_flip_weights(w, co, ci, C.c_void_p(self.wt.data_ptr()), self._stream()))
        h, wd = self.hs[l]
        fn = L_.pyr3_dn_conv3x3_bf16 if self.tc else L_.pyr3_dn_conv3x3
        _check(fn(g[0], g[1], co, dst[0], dst[1], ci, self.n, h, wd, C.c_void_p(self.wt.data_ptr()), None, 0,
                  self._stream()))

    def _wgrad(self, src, ci, g, co, l, i):
        self.launches += 3
        dw, db = self._gw(i)
        h, wd = self.hs[l]
        fn = _lib.lib().pyr3_dn_conv3x3_wgrad_bf16 if self.tc else _lib.lib().pyr3_dn_conv3x3_wgrad
        _check(fn(src[0], src[1], ci, g[0], g[1], co, self.n, h, wd, dw, db, C.c_void_p(self.wsc.data_ptr()),
                  self.wsc_n, self._stream()))

    def _mask(self, g, y, c, l):
        self.launches += 1
        h, wd = self.hs[l]
        _check(_lib.lib().pyr3_dn_relu_mask(g[0], g[1], y[0], y[1], c, self.n, h * wd, self._stream()))

    # ---- passes
    def set_batch(self, x: np.ndarray, target: np.ndarray | None = None) -> None:
        self.x.copy_(self.t.from_numpy(np.ascontiguousarray(x, np.float32)))
        if target is not None:
            self.tgt.copy_(self.t.from_numpy(np.ascontiguousarray(target, np.float32)))

    def forward(self) -> None:
        L, ch, lib, st = self.L, self.chans, _lib.lib(), self._stream
        i = 0
        for l in range(L):
            if l > 0:
                e, h = self._e(l - 1), self.hs[l - 1]
                v = self._v(self.inp[l])
                _check(lib.pyr3_dn_pool2(e[0], e[1], v[0], v[1], ch[l - 1], self.n, h[0], h[1], 0, 0, st()))
                self.launches += 1
            cin = self.in_ch if l == 0 else ch[l - 1]
            self._conv(self._v(self.inp[l]), cin, self._v(self.a[l]), ch[l], l, i, True)
            self._conv(self._v(self.a[l]), ch[l], self._e(l), ch[l], l, i + 1, True)
            i += 2
        below = self._v(self.bottom)
        for l in range(L - 2, -1, -1):
            h = self.hs[l + 1]
            cv = self._v(self.cat[l])
            _check(lib.pyr3_dn_up2(below[0], below[1], cv[0], cv[1], ch[l + 1], self.n, h[0], h[1], 0, st()))
            self.launches += 1
            self._conv(cv, ch[l + 1] + ch[l], self._v(self.da[l]), ch[l], l, i, True)
            self._conv(self._v(self.da[l]), ch[l], self._v(self.d[l]), ch[l], l, i + 1, True)
            below = self._v(self.d[l])
            i += 2
        o = self._v(self.out)
        self._conv(self._v(self.d[0]), ch[0], o, OUT_CH, 0, i, False)
        xv = self._v(self.x, IN_CH)
        _check(lib.pyr3_dn_add(o[0], o[1], xv[0], xv[1], OUT_CH, self.n, self.h * self.w, st()))
        self.launches += 1

    def loss_and_grad(self) -> None:
        """MSE of out against the target; its gradient into gout (loss stays
        on the device until read_loss)."""
        self.loss.zero_()
        self.launches += 1
        _check(_lib.lib().pyr3_dn_mse(C.c_void_p(self.out.data_ptr()), C.c_void_p(self.tgt.data_ptr()),
                                      self.out.numel(), C.c_void_p(self.gout.data_ptr()),
                                      C.c_void_p(self.loss.data_ptr()), self._stream()))

    def read_loss(self) -> float:
        return float(self.loss.item()) / self.out.numel()

    def backward(self) -> None:
        L, ch, lib, st = self.L, self.chans, _lib.lib(), self._stream
        last = len(self.shapes) - 1
        self._wgrad(self._v(self.d[0]), ch[0], self._v(self.gout), OUT_CH, 0, last)
        self._dgrad(self._v(self.gout), OUT_CH, self._v(self.gd[0]), ch[0], 0, last)
        for l in range(0, L - 1):
            i = 2 * L + 2 * (L - 2 - l)
            gd = self._v(self.gd[l])
            self._mask(gd, self._v(self.d[l]), ch[l], l)
            self._wgrad(self._v(self.da[l]), ch[l], gd, ch[l], l, i + 1)
            gt = self._v(self.gtmp[l])
            self._dgrad(gd, ch[l], gt, ch[l], l, i + 1)
            self._mask(gt, self._v(self.da[l]), ch[l], l)
            self._wgrad(self._v(self.cat[l]), ch[l + 1] + ch[l], gt, ch[l], l, i)
            gc = self._v(self.gcat[l])
            self._dgrad(gt, ch[l], gc, ch[l + 1] + ch[l], l, i)
            dst = self._v(self.gd[l + 1]) if l + 1 <= L - 2 else self._v(self.gbottom)
            h = self.hs[l + 1]
            _check(lib.pyr3_dn_up2(gc[0], gc[1], dst[0], dst[1], ch[l + 1], self.n, h[0], h[1], 1, st()))
            self.launches += 1
        for l in range(L - 1, -1, -1):
            i = 2 * l
            ge = self._ge(l)  # skip gradient + pooled gradient already accumulated
            self._mask(ge, self._e(l), ch[l], l)
            self._wgrad(self._v(self.a[l]), ch[l], ge, ch[l], l, i + 1)
            ga = self._v(self.gtmp[l])
            self._dgrad(ge, ch[l], ga, ch[l], l, i + 1)
            self._mask(ga, self._v(self.a[l]), ch[l], l)
            cin = self.in_ch if l == 0 else ch[l - 1]
            self._wgrad(self._v(self.inp[l]), cin, ga, ch[l], l, i)
            if l > 0:
                gi = self._v(self.ginp[l])
                self._dgrad(ga, ch[l], gi, cin, l, i)
                h = self.hs[l - 1]
                dst = self._ge(l - 1)
                _check(lib.pyr3_dn_pool2(gi[0], gi[1], dst[0], dst[1], ch[l - 1], self.n, h[0], h[1], 1, 1, st()))
                self.launches += 1

    def capture(self) -> None:
        """Record forward, loss and backward as one CUDA graph, so that a
        training step is one graph launch plus the Adam kernel instead of
        ~130 separate launches from Python.  Every captured kernel is this
        library's; replay() reruns them on whatever x and tgt hold."""
        t = self.t
        side = t.cuda.Stream(self.dev)
        side.wait_stream(t.cuda.current_stream(self.dev))
        with t.cuda.stream(side):  # every kernel runs once before capture
            self.forward()
            self.loss_and_grad()
            self.backward()
        t.cuda.current_stream(self.dev).wait_stream(side)
        self.graph = t.cuda.CUDAGraph()
        n0 = self.launches
        with t.cuda.graph(self.graph):
            self.forward()
            self.loss_and_grad()
            self.backward()
        self.graph_launches = self.launches - n0

    def replay(self) -> None:
        """forward + loss_and_grad + backward from the captured graph."""
        self.graph.replay()
        self.launches += self.graph_launches

    def step(self, lr: float = 1e-3, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8) -> None:
        self.steps += 1
        self.launches += 1
        _check(_lib.lib().pyr3_dn_adam(C.c_void_p(self.p.data_ptr()), C.c_void_p(self.g.data_ptr()),
                                       C.c_void_p(self.m.data_ptr()), C.c_void_p(self.v.data_ptr()),
                                       self.p.numel(), lr, b1, b2, eps, self.steps, self._stream()))

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy()

    def grads(self) -> np.ndarray:
        return self.g.cpu().numpy()

    def output(self) -> np.ndarray:
        return self.out.cpu().numpy()


def init_params(chans=CHANS, seed: int = 0, in_ch: int = IN_CH) -> np.ndarray:
    """He-normal weights, zero biases; the last conv starts at zero, so the
    untrained network returns the noisy image."""
    rng = np.random.default_rng(seed)
    parts = []
    shapes = layer_shapes(chans, in_ch)
    for i, (co, ci) in enumerate(shapes):
        std = 0.0 if i == len(shapes) - 1 else np.sqrt(2.0 / (ci * 9))
        parts += [rng.normal(0.0, 1.0, co * ci * 9) * std, np.zeros(co)]
    return np.concatenate(parts).astype(np.float32)


# Density-estimation setting the radius feature is computed with when the
# genome sets none (the plain_small configuration's 9 / 0 / 0.4).
FEATURE_DE = {"maxRad": 9.0, "minRad": 0.0, "curve": 0.4}


def features(renderer, genome, samples: int) -> np.ndarray:
    """(IN_CH + OUT_CH) x H x W input of the renderer's current histogram:
    the 8 feature channels, then the noisy tonemapped RGB."""
    img = renderer.present(genome, samples, fmt="f32", force_de_off=True).astype(np.float32)  # H x W x 4
    alpha = renderer.present(genome, samples, fmt="f32", force_de_off=True, transparent=True)[..., 3]
    hist, _, _ = renderer.read_histogram()
    os_, H, W = renderer.oversample, renderer.height, renderer.width
    h = hist.astype(np.float64).reshape(H, os_, W, os_, 4).sum(axis=(1, 3))
    hits = h[..., 3] / 255.0
    f = np.empty((IN_CH + OUT_CH, H, W), np.float32)
    f[0] = np.log1p(hits)
    with np.errstate(invalid="ignore", divide="ignore"):
        for c in range(3):
            f[1 + c] = np.where(h[..., 3] > 0, h[..., c] / np.maximum(h[..., 3], 1.0), 0.0)
    f[4] = alpha
    f[5] = hits * (W * H) / max(float(samples), 1.0)
    lum = img[..., 0] * 0.299 + img[..., 1] * 0.587 + img[..., 2] * 0.114
    pad = np.pad(lum.astype(np.float64), 1, mode="edge")
    win = np.stack([pad[dy:dy + H, dx:dx + W] for dy in range(3) for dx in range(3)])
    f[6] = win.var(axis=0)
    de = genome.density or FEATURE_DE
    mx, mn = de["maxRad"], de["minRad"]
    rad = np.clip(mx / np.power(hits + 1.0, de["curve"]), mn, mx)
    f[7] = np.where(hits > 0, rad / max(mx, 1e-6), 0.0)
    f[IN_CH:] = img[..., :3].transpose(2, 0, 1)
    return f


def target(renderer, genome, samples: int) -> np.ndarray:
    img = renderer.present(genome, samples, fmt="f32").astype(np.float32)
    return np.ascontiguousarray(img[..., :3].transpose(2, 0, 1))


def ssim(a: np.ndarray, b: np.ndarray) -> float:
    """Mean SSIM (Wang et al. 2004: 11x11 Gaussian window, sigma 1.5,
    K1 = 0.01, K2 = 0.03, dynamic range 1) over images and channels of
    N x C x H x W arrays in 0..1."""
    from scipy.ndimage import gaussian_filter

    c1, c2 = 0.01 ** 2, 0.03 ** 2
    vals = []
    for x, y in zip(a.reshape(-1, *a.shape[-2:]).astype(np.float64), b.reshape(-1, *b.shape[-2:]).astype(np.float64)):
        f = lambda z: gaussian_filter(z, 1.5, truncate=3.5)  # noqa: E731  (11-tap window)
        mx, my = f(x), f(y)
        sxx, syy, sxy = f(x * x) - mx * mx, f(y * y) - my * my, f(x * y) - mx * my
        vals.append(float((((2 * mx * my + c1) * (2 * sxy + c2)) /
                           ((mx * mx + my * my + c1) * (sxx + syy + c2))).mean()))
    return float(np.mean(vals))


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    mse = float(((a.astype(np.float64) - b) ** 2).mean())
    return 10.0 * np.log10(1.0 / max(mse, 1e-20))


def make_dataset(genomes, spp_in: float = 25.0, spp_target: float = 2000.0, seed: int = 0):
    """(inputs N x 11 x H x W, targets N x 3 x H x W) from renders of each
    genome at spp_in and spp_target samples per pixel (one renderer)."""
    from . import renderer as R

    W, H = genomes[0].size
    r = R.create_renderer(W, H, 1)
    xs, ts = [], []
    for i, g in enumerate(genomes):
        for spp, out in ((spp_in, xs), (spp_target, ts)):
            w, it, samples = R.compute_dispatch(spp, W, H)
            r.reset(g)
            r.iterate(g, seed + 7919 * i + (0 if spp == spp_in else 1), w, it)
            out.append(features(r, g, samples) if out is xs else target(r, g, samples))
    r.destroy()
    return np.stack(xs), np.stack(ts)


def train(xs, ts, steps: int = 300, batch: int = 8, crop: int = 128, lr: float = 1e-3, seed: int = 0,
          chans=CHANS, params=None, in_ch: int = IN_CH, lr_end: float | None = None):
    """Adam on random crops of (xs, ts), all on the device; the learning
    rate falls linearly from lr to lr_end over the steps when lr_end is
    given.  Returns (net, losses, device ms of the training steps)."""
    import torch

    rng = np.random.default_rng(seed)
    dev = torch.device("cuda", 0)
    X = torch.tensor(xs, device=dev)
    T = torch.tensor(ts, device=dev)
    n, _, H, W = xs.shape
    net = UNet(batch, crop, crop, init_params(chans, seed, in_ch) if params is None else params, chans=chans,
               in_ch=in_ch)
    net.capture()
    net.launches = 0
    losses = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for s in range(steps):
        idx = rng.integers(0, n, batch)
        ys, xo = rng.integers(0, H - crop + 1, batch), rng.integers(0, W - crop + 1, batch)
        for j in range(batch):
            net.x[j].copy_(X[idx[j], :, ys[j]:ys[j] + crop, xo[j]:xo[j] + crop])
            net.tgt[j].copy_(T[idx[j], :, ys[j]:ys[j] + crop, xo[j]:xo[j] + crop])
        net.replay()
        net.step(lr=lr if lr_end is None else lr + (lr_end - lr) * s / max(1, steps - 1))
        if s % 25 == 0 or s == steps - 1:
            losses.append((s, net.read_loss()))
    e1.record()
    e1.synchronize()
    return net, losses, e0.elapsed_time(e1)


def evaluate(params, xs, ts, chans=CHANS, tensor_cores: bool = True, in_ch: int = IN_CH):
    """(PSNR of the noisy input, PSNR of the denoised output) against the
    targets, over all images, and the denoised images."""
    n, _, H, W = xs.shape
    net = UNet(n, H, W, params, chans=chans, tensor_cores=tensor_cores, in_ch=in_ch)
    net.set_batch(xs, ts)
    net.forward()
    out = np.clip(net.output(), 0.0, 1.0)
    return psnr(np.clip(xs[:, IN_CH:IN_CH + OUT_CH], 0.0, 1.0), ts), psnr(out, ts), out


def plain_quality(genomes, targets, spps, seed: int = 99):
    """PSNR against `targets` of plain renders of `genomes` at each spp in
    `spps`, with the device time of those renders: [(spp, psnr, ms)]."""
    from . import renderer as R

    W, H = genomes[0].size
    r = R.create_renderer(W, H, 1)
    res = []
    for spp in spps:
        imgs, ms = [], 0.0
        for i, g in enumerate(genomes):
            w, it, samples = R.compute_dispatch(spp, W, H)
            r.reset(g)
            r.iterate(g, seed + i, w, it)
            ms += r.last_iterate_ms()
            imgs.append(target(r, g, samples))
        res.append((spp, psnr(np.stack(imgs), targets), ms))
    r.destroy()
    return res
