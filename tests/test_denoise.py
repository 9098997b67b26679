"""Learned denoiser.  CPU: the numpy oracle's layers and whole-U-Net gradient
against PyTorch-CPU autograd (the denoiser has no reference counterpart, so
autograd pins the oracle).  GPU: every CUDA layer against the oracle, then a
whole U-Net forward + backward (skip slices, pooling, upsampling, residual)
against the oracle, and Adam steps that lower the loss."""
import ctypes as C

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from oracle import denoise_ref as D

CH_SMALL = (4, 6, 8)


# ------------------------------------------------------------ CPU: oracle pins
def _torch_unet(params, x, chans):
    L = len(chans)
    in_ch = x.shape[1] - 3
    layers = [(torch.tensor(w, requires_grad=True), torch.tensor(b, requires_grad=True))
              for w, b in D.unpack(params, chans, in_ch)]
    xt = torch.tensor(x)
    e = []
    inp = xt[:, :in_ch]
    li = 0
    for l in range(L):
        if l > 0:
            inp = F.avg_pool2d(e[-1], 2)
        a = F.relu(F.conv2d(inp, layers[li][0], layers[li][1], padding=1))
        e.append(F.relu(F.conv2d(a, layers[li + 1][0], layers[li + 1][1], padding=1)))
        li += 2
    below = e[-1]
    for l in range(L - 2, -1, -1):
        cat = torch.cat([F.interpolate(below, scale_factor=2, mode="nearest"), e[l]], dim=1)
        da = F.relu(F.conv2d(cat, layers[li][0], layers[li][1], padding=1))
        below = F.relu(F.conv2d(da, layers[li + 1][0], layers[li + 1][1], padding=1))
        li += 2
    out = F.conv2d(below, layers[li][0], layers[li][1], padding=1) + xt[:, in_ch:in_ch + 3]
    return out, layers


def test_oracle_layers_match_torch_autograd():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 5, 8, 12))
    w = rng.normal(size=(7, 5, 3, 3))
    b = rng.normal(size=7)
    xt = torch.tensor(x, requires_grad=True)
    wt = torch.tensor(w, requires_grad=True)
    bt = torch.tensor(b, requires_grad=True)
    y = F.conv2d(xt, wt, bt, padding=1)
    g = rng.normal(size=y.shape)
    y.backward(torch.tensor(g))
    assert np.allclose(D.conv3x3(x, w, b), y.detach().numpy(), atol=1e-10)
    dw, db = D.conv3x3_wgrad(x, g)
    assert np.allclose(dw, wt.grad.numpy(), atol=1e-9) and np.allclose(db, bt.grad.numpy(), atol=1e-9)
    assert np.allclose(D.conv3x3_dgrad(g, w), xt.grad.numpy(), atol=1e-9)
    # pooling and upsampling adjoints
    xt2 = torch.tensor(x, requires_grad=True)
    p = F.avg_pool2d(xt2, 2)
    gp = rng.normal(size=p.shape)
    p.backward(torch.tensor(gp))
    assert np.allclose(D.pool2(x), p.detach().numpy()) and np.allclose(D.pool2_bwd(gp), xt2.grad.numpy())
    xt3 = torch.tensor(x, requires_grad=True)
    u = F.interpolate(xt3, scale_factor=2, mode="nearest")
    gu = rng.normal(size=u.shape)
    u.backward(torch.tensor(gu))
    assert np.allclose(D.up2(x), u.detach().numpy()) and np.allclose(D.up2_bwd(gu), xt3.grad.numpy())


def test_oracle_unet_gradient_matches_torch_autograd():
    rng = np.random.default_rng(1)
    params = D.init_params(CH_SMALL, seed=3)
    params[-(3 * 4 * 9 + 3):] = rng.normal(0.0, 0.1, 3 * 4 * 9 + 3)  # non-zero output conv
    x = rng.normal(size=(2, 8 + 3, 16, 16))  # 8 feature channels, then the noisy image
    tgt = rng.normal(size=(2, 3, 16, 16))
    out, cache = D.forward(params, x, CH_SMALL)
    loss, gout = D.mse(out, tgt)
    grad = D.backward(params, cache, gout, CH_SMALL)
    tout, layers = _torch_unet(params, x, CH_SMALL)
    tl = ((tout - torch.tensor(tgt)) ** 2).mean()
    tl.backward()
    tg = np.concatenate([np.concatenate([w.grad.numpy().ravel(), b.grad.numpy().ravel()]) for w, b in layers])
    assert np.allclose(out, tout.detach().numpy(), atol=1e-10)
    assert abs(loss / out.size - float(tl.detach())) < 1e-12
    assert np.allclose(grad, tg, rtol=1e-8, atol=1e-12)


def test_product_and_oracle_agree_on_architecture():
    from pyr3_b200 import denoise as DN

    assert DN.layer_shapes(CH_SMALL) == D.layer_shapes(CH_SMALL)
    assert DN.param_count() == sum(co * ci * 9 + co for co, ci in D.layer_shapes(DN.CHANS))
    assert 150_000 <= DN.param_count() <= 250_000


# ------------------------------------------------------------ GPU: CUDA vs oracle
def _dev(a):
    return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def _p(t, c0=0):
    return C.c_void_p(t.data_ptr() + 4 * c0 * t.shape[2] * t.shape[3])


def _bf16(a):
    """f32 rounded to bf16 (nearest even), as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _close(got, want, rtol=2e-4, atol=2e-5):
    got = got.detach().cpu().numpy().astype(np.float64) if isinstance(got, torch.Tensor) else got
    err = np.abs(got - want) - (atol + rtol * np.abs(want))
    assert float(err.max()) <= 0.0, float((np.abs(got - want)).max())


@pytest.mark.gpu
def test_cuda_layers_match_oracle():
    from pyr3_b200 import _lib

    L = _lib.lib()
    ck = _lib.check
    rng = np.random.default_rng(2)
    n, ci, co, h, w = 2, 11, 13, 20, 36  # tiles and channel groups with ragged edges
    x = rng.normal(size=(n, ci, h, w))
    wt = rng.normal(size=(co, ci, 3, 3)) * 0.2
    b = rng.normal(size=co)
    g = rng.normal(size=(n, co, h, w))
    xd, wd, bd, gd = _dev(x), _dev(wt), _dev(b), _dev(g)
    yd = torch.zeros((n, co, h, w), device="cuda")
    ck(L.pyr3_dn_conv3x3(_p(xd), ci * h * w, ci, _p(yd), co * h * w, co, n, h, w, C.c_void_p(wd.data_ptr()),
                         C.c_void_p(bd.data_ptr()), 1, None))
    torch.cuda.synchronize()
    _close(yd, D.conv3x3(x, wt, b, relu=True))
    dw = torch.zeros_like(wd)
    db = torch.zeros_like(bd)
    nsc = L.pyr3_dn_wgrad_scratch_floats(co, ci)
    sc = torch.zeros(nsc, device="cuda")
    with pytest.raises(Exception):  # too little scratch is refused
        ck(L.pyr3_dn_conv3x3_wgrad(_p(xd), ci * h * w, ci, _p(gd), co * h * w, co, n, h, w,
                                   C.c_void_p(dw.data_ptr()), C.c_void_p(db.data_ptr()), C.c_void_p(sc.data_ptr()),
                                   nsc - 1, None))
    ck(L.pyr3_dn_conv3x3_wgrad(_p(xd), ci * h * w, ci, _p(gd), co * h * w, co, n, h, w,
                               C.c_void_p(dw.data_ptr()), C.c_void_p(db.data_ptr()), C.c_void_p(sc.data_ptr()),
                               nsc, None))
    ref_dw, ref_db = D.conv3x3_wgrad(x, g)
    torch.cuda.synchronize()
    _close(dw, ref_dw, rtol=1e-4, atol=1e-3)
    _close(db, ref_db, rtol=1e-4, atol=1e-3)
    fl = torch.zeros_like(wd)
    ck(L.pyr3_dn_flip_weights(C.c_void_p(wd.data_ptr()), co, ci, C.c_void_p(fl.data_ptr()), None))
    dx = torch.zeros_like(xd)
    ck(L.pyr3_dn_conv3x3(_p(gd), co * h * w, co, _p(dx), ci * h * w, ci, n, h, w, C.c_void_p(fl.data_ptr()),
                         None, 0, None))
    torch.cuda.synchronize()
    _close(dx, D.conv3x3_dgrad(g, wt))
    # tensor-core weight gradient: the oracle on bf16-rounded operands, f32 sums
    for co2, ci2 in ((co, ci), (90, 40)):
        x2, g2 = rng.normal(size=(n, ci2, h, w)), rng.normal(size=(n, co2, h, w))
        x2d, g2d = _dev(x2), _dev(g2)
        dw2 = torch.zeros((co2, ci2, 3, 3), device="cuda")
        db2 = torch.zeros(co2, device="cuda")
        nsc2 = L.pyr3_dn_wgrad_scratch_floats(co2, ci2)
        sc2 = torch.zeros(nsc2, device="cuda")
        ck(L.pyr3_dn_conv3x3_wgrad_bf16(_p(x2d), ci2 * h * w, ci2, _p(g2d), co2 * h * w, co2, n, h, w,
                                        C.c_void_p(dw2.data_ptr()), C.c_void_p(db2.data_ptr()),
                                        C.c_void_p(sc2.data_ptr()), nsc2, None))
        torch.cuda.synchronize()
        rdw, rdb = D.conv3x3_wgrad(_bf16(x2), _bf16(g2))
        _close(dw2, rdw, rtol=1e-4, atol=1e-3)
        _close(db2, D.conv3x3_wgrad(x2, g2.astype(np.float32).astype(np.float64))[1], rtol=1e-4, atol=1e-3)
    # tensor-core convolution: the oracle on bf16-rounded operands, f32 sums
    for co2 in (co, 40, 90):
        w2 = rng.normal(size=(co2, ci, 3, 3)) * 0.2
        b2 = rng.normal(size=co2)
        w2d, b2d = _dev(w2), _dev(b2)
        y2 = torch.zeros((n, co2, h, w), device="cuda")
        ck(L.pyr3_dn_conv3x3_bf16(_p(xd), ci * h * w, ci, _p(y2), co2 * h * w, co2, n, h, w,
                                  C.c_void_p(w2d.data_ptr()), C.c_void_p(b2d.data_ptr()), 1, None))
        torch.cuda.synchronize()
        want = D.conv3x3(_bf16(x), _bf16(w2), b2.astype(np.float32).astype(np.float64), relu=True)
        _close(y2, want, rtol=1e-4, atol=1e-4)
    # pool / upsample on a channel slice of a wider tensor (stride != channels * hw)
    big = _dev(rng.normal(size=(n, 7, h, w)))
    src = big.cpu().numpy().astype(np.float64)[:, 2:5]
    po = torch.zeros((n, 3, h // 2, w // 2), device="cuda")
    ck(L.pyr3_dn_pool2(_p(big, 2), 7 * h * w, _p(po), 3 * (h // 2) * (w // 2), 3, n, h, w, 0, 0, None))
    torch.cuda.synchronize()
    _close(po, D.pool2(src))
    acc = torch.ones((n, 3, h, w), device="cuda")
    ck(L.pyr3_dn_pool2(_p(po), 3 * (h // 2) * (w // 2), _p(acc), 3 * h * w, 3, n, h, w, 1, 1, None))
    torch.cuda.synchronize()
    _close(acc, 1.0 + D.pool2_bwd(D.pool2(src)))
    up = torch.zeros((n, 3, 2 * h, 2 * w), device="cuda")
    ck(L.pyr3_dn_up2(_p(big, 2), 7 * h * w, _p(up), 3 * 4 * h * w, 3, n, h, w, 0, None))
    back = torch.zeros((n, 3, h, w), device="cuda")
    ck(L.pyr3_dn_up2(_p(up), 3 * 4 * h * w, _p(back), 3 * h * w, 3, n, h, w, 1, None))
    torch.cuda.synchronize()
    _close(up, D.up2(src))
    _close(back, D.up2_bwd(D.up2(src)))
    # ReLU mask, add, MSE, Adam
    gm = _dev(g)
    ck(L.pyr3_dn_relu_mask(_p(gm), co * h * w, _p(yd), co * h * w, co, n, h * w, None))
    torch.cuda.synchronize()
    _close(gm, g * (yd.cpu().numpy() > 0))  # the mask of the device's own ReLU output
    pred, tgt = rng.normal(size=(n, 3, h, w)), rng.normal(size=(n, 3, h, w))
    pd, td, gr = _dev(pred), _dev(tgt), torch.zeros((n, 3, h, w), device="cuda")
    loss = torch.zeros(1, device="cuda")
    ck(L.pyr3_dn_mse(C.c_void_p(pd.data_ptr()), C.c_void_p(td.data_ptr()), pd.numel(), C.c_void_p(gr.data_ptr()),
                     C.c_void_p(loss.data_ptr()), None))
    ref_loss, ref_g = D.mse(pred, tgt)
    torch.cuda.synchronize()
    _close(gr, ref_g)
    assert abs(float(loss.item()) - ref_loss) <= 1e-4 * ref_loss
    p0, g0 = rng.normal(size=1000), rng.normal(size=1000)
    pdv, gdv, m, v = _dev(p0), _dev(g0), torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    rp, rm, rv = p0.copy(), np.zeros(1000), np.zeros(1000)
    for step in (1, 2, 3):
        ck(L.pyr3_dn_adam(C.c_void_p(pdv.data_ptr()), C.c_void_p(gdv.data_ptr()), C.c_void_p(m.data_ptr()),
                          C.c_void_p(v.data_ptr()), 1000, 1e-2, 0.9, 0.999, 1e-8, step, None))
        rp, rm, rv = D.adam(rp, g0, rm, rv, step, lr=1e-2)
    torch.cuda.synchronize()
    _close(pdv, rp, rtol=1e-5, atol=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("n,ci,co,h,w", [(1, 40, 16, 48, 130), (3, 8, 96, 17, 256), (2, 88, 40, 8, 8)])
def test_tensor_core_convolution_tiles_match_oracle(n, ci, co, h, w):
    """The tcgen05 convolution with several 128-position tiles per CTA
    sharing one staged window (wide rows: 130 and 256 columns; a tail CTA
    whose last tiles lie past the image) and with one tile (an 8 x 8
    level): the oracle on bf16-rounded operands, f32 sums."""
    from pyr3_b200 import _lib

    rng = np.random.default_rng(ci + co + w)
    x = rng.normal(size=(n, ci, h, w))
    wt = rng.normal(size=(co, ci, 3, 3)) * 0.2
    b = rng.normal(size=co)
    xd, wd, bd = _dev(x), _dev(wt), _dev(b)
    y = torch.zeros((n, co, h, w), device="cuda")
    _lib.check(_lib.lib().pyr3_dn_conv3x3_bf16(_p(xd), ci * h * w, ci, _p(y), co * h * w, co, n, h, w,
                                               C.c_void_p(wd.data_ptr()), C.c_void_p(bd.data_ptr()), 1, None))
    torch.cuda.synchronize()
    want = D.conv3x3(_bf16(x), _bf16(wt), b.astype(np.float32).astype(np.float64), relu=True)
    _close(y, want, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("in_ch", [8, 11])
def test_cuda_unet_forward_backward_matches_oracle(in_ch):
    """The whole U-Net's output and parameter gradient against the numpy
    oracle, reading the 8 feature channels, or those and the noisy image
    (11); the output is added to the noisy image either way."""
    from pyr3_b200 import denoise as DN

    chans = (8, 12, 16)
    rng = np.random.default_rng(4)
    params = DN.init_params(chans, seed=5, in_ch=in_ch)
    params[-(3 * 8 * 9 + 3):] = rng.normal(0.0, 0.05, 3 * 8 * 9 + 3)
    n, h, w = 2, 32, 48
    x = rng.normal(size=(n, DN.IN_CH + DN.OUT_CH, h, w))  # features, then the noisy image
    tgt = rng.normal(size=(n, 3, h, w))
    net = DN.UNet(n, h, w, params, chans=chans, tensor_cores=False, in_ch=in_ch)
    net.set_batch(x, tgt)
    net.forward()
    net.loss_and_grad()
    net.backward()
    torch.cuda.synchronize()
    out, cache = D.forward(params.astype(np.float64), x, chans, in_ch=in_ch)
    loss, gout = D.mse(out, tgt)
    grad = D.backward(params.astype(np.float64), cache, gout, chans)
    _close(net.output(), out, rtol=1e-4, atol=1e-4)
    assert abs(net.read_loss() - loss / out.size) <= 1e-4 * loss / out.size
    got = net.grads().astype(np.float64)
    scale = np.abs(grad).max()
    assert float(np.abs(got - grad).max()) <= 1e-3 * scale, float(np.abs(got - grad).max() / scale)
    # the captured graph reruns the same kernels: the same gradient, bit for bit
    net.capture()
    net.g.zero_()
    net.replay()
    torch.cuda.synchronize()
    assert np.array_equal(net.grads(), got.astype(np.float32))
    # the tensor-core network (bf16 operands, f32 accumulation) stays close
    tcn = DN.UNet(n, h, w, params, chans=chans, tensor_cores=True, in_ch=in_ch)
    tcn.set_batch(x, tgt)
    tcn.forward()
    tcn.loss_and_grad()
    tcn.backward()
    torch.cuda.synchronize()
    o2 = tcn.output().astype(np.float64)
    assert float(np.abs(o2 - out).max()) <= 3e-2 * float(np.abs(out).max())
    g2 = tcn.grads().astype(np.float64)
    cos = float(g2 @ grad / (np.linalg.norm(g2) * np.linalg.norm(grad)))
    assert cos >= 0.99, cos


@pytest.mark.gpu
def test_adam_training_lowers_the_loss():
    from pyr3_b200 import denoise as DN

    rng = np.random.default_rng(6)
    n, h, w = 2, 32, 32
    clean = rng.uniform(0.0, 1.0, (n, 3, 1, 1)) * np.ones((n, 3, h, w))
    noisy = clean + rng.normal(0.0, 0.2, clean.shape)
    x = np.concatenate([noisy, rng.normal(size=(n, 5, h, w)), noisy], axis=1)
    net = DN.UNet(n, h, w, DN.init_params(seed=7))
    net.set_batch(x, clean)
    losses = []
    for _ in range(60):
        net.forward()
        net.loss_and_grad()
        net.backward()
        net.step(lr=2e-3)
        losses.append(net.read_loss())
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
