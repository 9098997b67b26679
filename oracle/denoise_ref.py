"""CPU oracle of the learned denoiser (test infrastructure only: tests/ use it
as the checker; the product never imports it).

The denoiser has no counterpart in the reference, so its parity is pinned
differently: every layer and the whole U-Net's gradient are checked here
against PyTorch-CPU autograd (tests/test_denoise.py), and the CUDA layers
are checked against this oracle.

Tensors are NCHW float64 numpy arrays.  The U-Net: L levels of channels
chans[0..L-1]; encoder level l = two 3x3 conv + ReLU (input: the 8 feature
channels, or the 2x2 average pool of level l-1); decoder level l (L-2 .. 0)
= nearest 2x upsample of the level below, concatenated with the encoder's
level-l output (upsampled channels first), then two 3x3 conv + ReLU; a last
3x3 conv to 3 channels, added to input channels 0..2.  Parameters are one
flat vector: per conv, in layer order, weight [co][ci][3][3] then bias[co].
"""
from __future__ import annotations

import numpy as np


def conv3x3(x, w, b=None, relu=False):
    n, ci, h, wd = x.shape
    co = w.shape[0]
    xp = np.zeros((n, ci, h + 2, wd + 2))
    xp[:, :, 1:-1, 1:-1] = x
    out = np.zeros((n, co, h, wd))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("oc,nchw->nohw", w[:, :, ky, kx], xp[:, :, ky:ky + h, kx:kx + wd])
    if b is not None:
        out += b[None, :, None, None]
    return np.maximum(out, 0.0) if relu else out


def conv3x3_wgrad(x, dout):
    n, ci, h, wd = x.shape
    xp = np.zeros((n, ci, h + 2, wd + 2))
    xp[:, :, 1:-1, 1:-1] = x
    dw = np.zeros((dout.shape[1], ci, 3, 3))
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("nohw,nchw->oc", dout, xp[:, :, ky:ky + h, kx:kx + wd])
    return dw, dout.sum(axis=(0, 2, 3))


def flip_weights(w):
    """[co][ci][ky][kx] -> [ci][co][2-ky][2-kx]."""
    return np.ascontiguousarray(w.transpose(1, 0, 2, 3)[:, :, ::-1, ::-1])


def conv3x3_dgrad(dout, w):
    return conv3x3(dout, flip_weights(w))


def pool2(x):
    n, c, h, w = x.shape
    return x.reshape(n, c, h // 2, 2, w // 2, 2).mean(axis=(3, 5))


def pool2_bwd(g):
    return np.repeat(np.repeat(g, 2, axis=2), 2, axis=3) * 0.25


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)


def up2_bwd(g):
    n, c, h, w = g.shape
    return g.reshape(n, c, h // 2, 2, w // 2, 2).sum(axis=(3, 5))


def mse(pred, target):
    d = pred - target
    return float((d * d).sum()), 2.0 * d / d.size


def adam(p, g, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    p = p - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return p, m, v


def layer_shapes(chans, in_ch=8, out_ch=3):
    """(co, ci) of every conv in parameter order."""
    L = len(chans)
    shapes = []
    for l in range(L):
        ci = in_ch if l == 0 else chans[l - 1]
        shapes += [(chans[l], ci), (chans[l], chans[l])]
    for l in range(L - 2, -1, -1):
        shapes += [(chans[l], chans[l + 1] + chans[l]), (chans[l], chans[l])]
    shapes.append((out_ch, chans[0]))
    return shapes


def unpack(params, chans, in_ch=8, out_ch=3):
    out, o = [], 0
    for co, ci in layer_shapes(chans, in_ch, out_ch):
        w = params[o:o + co * ci * 9].reshape(co, ci, 3, 3)
        o += co * ci * 9
        b = params[o:o + co]
        o += co
        out.append((w, b))
    return out


def forward(params, x, chans, in_ch=None):
    """Returns (output, cache) for unet_backward.  x holds the feature
    channels followed by the three channels of the noisy image that the
    last convolution's output is added to; the first convolution reads
    channels 0..in_ch-1 (default: the features only)."""
    L = len(chans)
    in_ch = x.shape[1] - 3 if in_ch is None else in_ch
    layers = unpack(params, chans, in_ch)
    cache = {"x": x, "in_ch": in_ch, "inp": [], "a": [], "e": [], "cat": [], "da": [], "d": {}}
    inp = x[:, :in_ch]
    li = 0
    for l in range(L):
        if l > 0:
            inp = pool2(cache["e"][l - 1])
        cache["inp"].append(inp)
        a = conv3x3(inp, *layers[li], relu=True)
        e = conv3x3(a, *layers[li + 1], relu=True)
        li += 2
        cache["a"].append(a)
        cache["e"].append(e)
    below = cache["e"][L - 1]
    cats, das = {}, {}
    for l in range(L - 2, -1, -1):
        cat = np.concatenate([up2(below), cache["e"][l]], axis=1)
        da = conv3x3(cat, *layers[li], relu=True)
        d = conv3x3(da, *layers[li + 1], relu=True)
        li += 2
        cats[l], das[l], cache["d"][l] = cat, da, d
        below = d
    cache["cat"], cache["da"] = cats, das
    out = conv3x3(cache["d"][0], *layers[li]) + x[:, x.shape[1] - 3:]
    return out, cache


def backward(params, cache, gout, chans):
    """Gradient of the loss w.r.t. the flat parameters, given d loss / d out."""
    L = len(chans)
    layers = unpack(params, chans, cache["in_ch"])
    grads = [None] * len(layers)
    lo = len(layers) - 1
    dw, db = conv3x3_wgrad(cache["d"][0], gout)
    grads[lo] = (dw, db)
    g = conv3x3_dgrad(gout, layers[lo][0])
    gskip = {}
    # decoder, top level first (reverse of the forward order)
    for l in range(0, L - 1):
        li = 2 * L + 2 * (L - 2 - l)
        g = g * (cache["d"][l] > 0)
        grads[li + 1] = conv3x3_wgrad(cache["da"][l], g)
        g = conv3x3_dgrad(g, layers[li + 1][0]) * (cache["da"][l] > 0)
        grads[li] = conv3x3_wgrad(cache["cat"][l], g)
        gcat = conv3x3_dgrad(g, layers[li][0])
        cu = chans[l + 1]
        gskip[l] = gcat[:, cu:]
        g = up2_bwd(gcat[:, :cu])
    ge = g  # gradient of the bottom level's output
    for l in range(L - 1, -1, -1):
        if l < L - 1:
            ge = gskip[l] + gpool
        li = 2 * l
        ge = ge * (cache["e"][l] > 0)
        grads[li + 1] = conv3x3_wgrad(cache["a"][l], ge)
        ga = conv3x3_dgrad(ge, layers[li + 1][0]) * (cache["a"][l] > 0)
        grads[li] = conv3x3_wgrad(cache["inp"][l], ga)
        if l > 0:
            gpool = pool2_bwd(conv3x3_dgrad(ga, layers[li][0]))
    return np.concatenate([np.concatenate([dw.ravel(), db.ravel()]) for dw, db in grads])


def init_params(chans, in_ch=8, out_ch=3, seed=0):
    """He-normal weights, zero biases; the last conv starts at zero so the
    untrained network returns its input's colour channels."""
    rng = np.random.default_rng(seed)
    parts = []
    shapes = layer_shapes(chans, in_ch, out_ch)
    for i, (co, ci) in enumerate(shapes):
        std = 0.0 if i == len(shapes) - 1 else np.sqrt(2.0 / (ci * 9))
        parts += [rng.normal(0.0, 1.0, co * ci * 9) * std, np.zeros(co)]
    return np.concatenate(parts)
