"""Tensor-core 3x3 convolutions (forward, data gradient, weight gradient)
through the C ABI against torch-CPU float32 convolutions of the same
bf16-rounded operands.  Outputs are bf16 (forward, dgrad): tolerance 1 bf16
ulp relative plus a small absolute term; wgrad is fp32: 1e-4 relative to the
gradient's scale."""

import numpy as np
import pytest
import torch
import torch.nn.functional as Fn

from igm_b200 import _lib as L

pytestmark = pytest.mark.gpu


def to_rc(x_nchw):
    """[B, C, H, W] -> row-chunked [B, H, C/8, W, 8]"""
    B, Cc, H, W = x_nchw.shape
    return x_nchw.reshape(B, Cc // 8, 8, H, W).permute(0, 3, 1, 4, 2).contiguous()


def from_rc(x):
    B, H, C8, W, E = x.shape
    return x.permute(0, 2, 4, 1, 3).reshape(B, C8 * E, H, W)


def bf(t):
    return t.to(torch.bfloat16).to(torch.float32)


def pack_fwd(w_kkio, cin_t):
    """Keras kernel [3,3,cin,32] -> [kw][cin_t/8][kh][32][8] bf16."""
    kh, kw, cin, co = w_kkio.shape
    out = torch.zeros(3, cin_t // 8, 3, co, 8)
    for y in range(3):
        for x in range(3):
            for ci in range(cin):
                out[x, ci // 8, y, :, ci % 8] = w_kkio[y, x, ci, :]
    return out.to(torch.bfloat16).contiguous()


def pack_bwd(w_kkio):
    """Flipped, transposed dgrad pack: [2-kw][co/8][2-kh][ci][co%8] bf16."""
    out = torch.zeros(3, 4, 3, 32, 8)
    for y in range(3):
        for x in range(3):
            for co in range(32):
                out[2 - x, co // 8, 2 - y, :, co % 8] = w_kkio[y, x, :, co]
    return out.to(torch.bfloat16).contiguous()


def keras_to_torch(w):
    return w.permute(3, 2, 0, 1)  # [co, ci, kh, kw]


SHAPES = [(1, 4, 128, 32), (1, 9, 200, 32), (2, 7, 37, 32), (1, 13, 1000, 32), (1, 1, 5, 32), (3, 6, 129, 16),
          (1, 33, 300, 16)]


@pytest.mark.parametrize("B,H,W,cin", SHAPES)
def test_conv_forward(B, H, W, cin):
    g = torch.Generator().manual_seed(H * 1000 + W)
    x = bf(torch.randn(B, cin, H, W, generator=g))
    cin_real = cin if cin == 32 else 5
    if cin == 16:
        x[:, 5:] = 0
    w = torch.randn(3, 3, cin_real, 32, generator=g) * (1.0 / np.sqrt(9 * cin_real))
    b = torch.randn(32, generator=g) * 0.1
    ref = Fn.leaky_relu(Fn.conv2d(x[:, :cin_real], bf(keras_to_torch(w)), b, padding=1), 0.01)
    xd = to_rc(x).to(torch.bfloat16).cuda()
    wp = pack_fwd(w, cin).cuda()
    y = torch.empty((B, H, 4, W, 8), dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    bd = b.cuda()
    rc = L.lib().igm_conv3x3(0, B, H, W, cin, xd.data_ptr(), wp.data_ptr(), bd.data_ptr(), None,
                             y.data_ptr(), None, 0, 0.01, err.data_ptr(), L.stream_ptr())
    L.check(rc)
    out = from_rc(y.float().cpu())
    assert int(err.item()) == 0
    np.testing.assert_allclose(out.numpy(), ref.numpy(), rtol=8e-3, atol=2e-3 * float(ref.abs().max()))


@pytest.mark.parametrize("B,H,W", [(1, 8, 128), (2, 11, 173), (1, 5, 1000)])
def test_conv_dgrad(B, H, W):
    g = torch.Generator().manual_seed(B * 100 + H)
    gout = bf(torch.randn(B, 32, H, W, generator=g))
    aprev = bf(torch.randn(B, 32, H, W, generator=g))
    w = torch.randn(3, 3, 32, 32, generator=g) * (1.0 / np.sqrt(288))
    dx = torch.nn.grad.conv2d_input((B, 32, H, W), bf(keras_to_torch(w)), gout, padding=1)
    ref = dx * torch.where(aprev > 0, 1.0, 0.01)
    y = torch.empty((B, H, 4, W, 8), dtype=torch.bfloat16, device="cuda")
    dbp = torch.zeros((148, 32), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    gd = to_rc(gout).to(torch.bfloat16).cuda()
    wd = pack_bwd(w).cuda()
    ad = to_rc(aprev).to(torch.bfloat16).cuda()
    rc = L.lib().igm_conv3x3(1, B, H, W, 32, gd.data_ptr(), wd.data_ptr(), None, ad.data_ptr(),
                             y.data_ptr(), dbp.data_ptr(), 148, 0.01, err.data_ptr(), L.stream_ptr())
    L.check(rc)
    out = from_rc(y.float().cpu())
    assert int(err.item()) == 0
    np.testing.assert_allclose(out.numpy(), ref.numpy(), rtol=8e-3, atol=2e-3 * float(ref.abs().max()))
    db = dbp.sum(0).cpu().numpy()
    np.testing.assert_allclose(db, ref.sum((0, 2, 3)).numpy(), rtol=1e-3, atol=1e-3 * float(ref.abs().sum((0, 2, 3)).max()))


@pytest.mark.parametrize("B,H,W,cin", [(1, 8, 128, 32), (2, 9, 150, 32), (1, 6, 1000, 32), (2, 10, 77, 16)])
def test_conv_wgrad(B, H, W, cin):
    g = torch.Generator().manual_seed(H * 7 + W)
    x = bf(torch.randn(B, cin, H, W, generator=g))
    cin_real = 32 if cin == 32 else 5
    if cin == 16:
        x[:, 5:] = 0
    gout = bf(torch.randn(B, 32, H, W, generator=g))
    ref = torch.nn.grad.conv2d_weight(x[:, :cin_real], (32, cin_real, 3, 3), gout, padding=1)  # [co, ci, kh, kw]
    ref_k = ref.permute(2, 3, 1, 0).contiguous()  # Keras [kh, kw, ci, co]
    npart = 37
    part = torch.empty((npart, int(L.lib().igm_conv3x3_wgrad_partial_len(cin))), device="cuda")
    out = torch.empty((3, 3, cin_real, 32), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    xd = to_rc(x).to(torch.bfloat16).cuda()
    gd = to_rc(gout).to(torch.bfloat16).cuda()
    rc = L.lib().igm_conv3x3_wgrad(B, H, W, cin, xd.data_ptr(), gd.data_ptr(), part.data_ptr(), npart,
                                   err.data_ptr(), L.stream_ptr())
    L.check(rc)
    L.check(L.lib().igm_cnn_wgrad_finish(part.data_ptr(), npart, cin_real, cin, out.data_ptr(), L.stream_ptr()))
    assert int(err.item()) == 0
    np.testing.assert_allclose(out.cpu().numpy(), ref_k.numpy(), rtol=1e-4, atol=1e-4 * float(ref_k.abs().max()))


@pytest.mark.parametrize("B,H,W,npart", [(1, 8, 128, 148), (2, 11, 173, 37), (1, 5, 1000, 148), (1, 1000, 1000, 148),
                                         (3, 4, 40, 148), (1, 2, 7, 5)])
def test_conv_backward_fused(B, H, W, npart):
    """igm_conv3x3_backward (both gradients of a 32-channel layer in one pass):
    the data gradient bit for bit as igm_conv3x3(IGM_CONV_DGRAD) writes it, the
    weight-gradient partials bit for bit as igm_conv3x3_wgrad's (the same work
    items in the same order per CTA), the bias gradient to the rounding of its
    summation order, and both against torch-CPU float32."""
    g = torch.Generator().manual_seed(B * 1000 + H + W)
    gout = bf(torch.randn(B, 32, H, W, generator=g))
    aprev = bf(torch.randn(B, 32, H, W, generator=g))
    w = torch.randn(3, 3, 32, 32, generator=g) * (1.0 / np.sqrt(288))
    lib, st = L.lib(), L.stream_ptr()
    gd = to_rc(gout).to(torch.bfloat16).cuda()
    ad = to_rc(aprev).to(torch.bfloat16).cuda()
    wd = pack_bwd(w).cuda()
    plen = int(lib.igm_conv3x3_wgrad_partial_len(32))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y1 = torch.empty((B, H, 4, W, 8), dtype=torch.bfloat16, device="cuda")
    db1 = torch.zeros((npart, 32), device="cuda")
    p1 = torch.full((npart, plen), float("nan"), device="cuda")
    L.check(lib.igm_conv3x3(1, B, H, W, 32, gd.data_ptr(), wd.data_ptr(), None, ad.data_ptr(), y1.data_ptr(),
                            db1.data_ptr(), npart, 0.01, err.data_ptr(), st))
    L.check(lib.igm_conv3x3_wgrad(B, H, W, 32, ad.data_ptr(), gd.data_ptr(), p1.data_ptr(), npart, err.data_ptr(), st))
    y2 = torch.empty_like(y1)
    db2 = torch.full((npart, 32), float("nan"), device="cuda")
    p2 = torch.full((npart, plen), float("nan"), device="cuda")
    L.check(lib.igm_conv3x3_backward(B, H, W, gd.data_ptr(), wd.data_ptr(), ad.data_ptr(), y2.data_ptr(),
                                     db2.data_ptr(), p2.data_ptr(), npart, 0.01, err.data_ptr(), None, None, None, None,
                                     st))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(y1, y2)
    assert torch.equal(p1, p2)
    assert bool(torch.isfinite(db2).all())
    s1, s2 = db1.sum(0).double(), db2.sum(0).double()
    assert float((s1 - s2).abs().max()) <= 1e-5 * float(s1.abs().max()) + 1e-6
    # against torch
    dx = torch.nn.grad.conv2d_input((B, 32, H, W), bf(keras_to_torch(w)), gout, padding=1)
    ref = dx * torch.where(aprev > 0, 1.0, 0.01)
    np.testing.assert_allclose(from_rc(y2.float().cpu()).numpy(), ref.numpy(), rtol=8e-3,
                               atol=2e-3 * float(ref.abs().max()))
    ref_w = torch.nn.grad.conv2d_weight(aprev, (32, 32, 3, 3), gout, padding=1).permute(2, 3, 1, 0).contiguous()
    out = torch.empty((3, 3, 32, 32), device="cuda")
    L.check(lib.igm_cnn_wgrad_finish(p2.data_ptr(), npart, 32, 32, out.data_ptr(), st))
    np.testing.assert_allclose(out.cpu().numpy(), ref_w.numpy(), rtol=1e-4, atol=1e-4 * float(ref_w.abs().max()))


@pytest.mark.parametrize("B,H,W,nl,pingpong", [(1, 8, 128, 1, True), (1, 37, 300, 3, True), (2, 11, 173, 4, False),
                                               (1, 1000, 1000, 15, True), (1, 1000, 1000, 15, False),
                                               (3, 5, 40, 2, True), (1, 200, 1000, 16, True)])
def test_conv_stack(B, H, W, nl, pingpong):
    """igm_conv3x3_stack: nl forward layers in one launch, bit for bit what nl
    igm_conv3x3 calls write, with the outputs alternating between two buffers
    or in one buffer per layer; a second call on the same flag buffer (the
    next epoch) gives the same result."""
    g = torch.Generator().manual_seed(B * 7 + H * 3 + W + nl)
    lib, st = L.lib(), L.stream_ptr()
    x = to_rc(bf(torch.randn(B, 32, H, W, generator=g))).to(torch.bfloat16).cuda()
    ws = [pack_fwd(torch.randn(3, 3, 32, 32, generator=g) * (1.3 / np.sqrt(288)), 32).cuda() for _ in range(nl)]
    bs = [(torch.randn(32, generator=g) * 0.1).cuda() for _ in range(nl)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ref, cur = [], x
    for k in range(nl):
        y = torch.empty_like(x)
        L.check(lib.igm_conv3x3(0, B, H, W, 32, cur.data_ptr(), ws[k].data_ptr(), bs[k].data_ptr(), None,
                                y.data_ptr(), None, 0, 0.01, err.data_ptr(), st))
        ref.append(y)
        cur = y
    bufs = [torch.full_like(x, float("nan")) for _ in range(2 if pingpong else nl)]
    outs = [bufs[k % 2] if pingpong else bufs[k] for k in range(nl)]
    P = __import__("ctypes").c_void_p
    flags = torch.zeros(int(lib.igm_conv3x3_stack_flags_len(B, H, W, nl)), dtype=torch.int32, device="cuda")
    for epoch in (1, 2):
        L.check(lib.igm_conv3x3_stack(B, H, W, nl, x.data_ptr(), (P * nl)(*[o.data_ptr() for o in outs]),
                                      (P * nl)(*[w.data_ptr() for w in ws]), (P * nl)(*[b.data_ptr() for b in bs]),
                                      flags.data_ptr(), epoch, 0.01, err.data_ptr(), st))
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        assert bool((flags == epoch).all())
        assert torch.equal(outs[-1], ref[-1])
        if not pingpong:
            for k in range(nl):
                assert torch.equal(outs[k], ref[k]), k


@pytest.mark.parametrize("B,H,W,npart", [(1, 8, 128, 148), (2, 37, 300, 23), (1, 1000, 1000, 148)])
def test_conv_backward_finishes_the_previous_layer(B, H, W, npart):
    """A fused backward call given the previous call's partial buffers also
    finishes them: the kernel gradient bit for bit as igm_cnn_wgrad_finish, the
    bias gradient as igm_reduce_partials; its own outputs are unchanged."""
    g = torch.Generator().manual_seed(B + H + W)
    lib, st = L.lib(), L.stream_ptr()
    mk = lambda: to_rc(bf(torch.randn(B, 32, H, W, generator=g))).to(torch.bfloat16).cuda()  # noqa: E731
    g1, x1, g2, x2 = mk(), mk(), mk(), mk()
    w1 = pack_bwd(torch.randn(3, 3, 32, 32, generator=g) * (1.0 / np.sqrt(288))).cuda()
    w2 = pack_bwd(torch.randn(3, 3, 32, 32, generator=g) * (1.0 / np.sqrt(288))).cuda()
    plen = int(lib.igm_conv3x3_wgrad_partial_len(32))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y1, y2, y2b = (torch.empty_like(g1) for _ in range(3))
    p1, p2, p2b = (torch.full((npart, plen), float("nan"), device="cuda") for _ in range(3))
    d1, d2, d2b = (torch.full((npart, 32), float("nan"), device="cuda") for _ in range(3))
    call = lambda gg, ww, xx, yy, dd, pp, *fin: L.check(lib.igm_conv3x3_backward(  # noqa: E731
        B, H, W, gg.data_ptr(), ww.data_ptr(), xx.data_ptr(), yy.data_ptr(), dd.data_ptr(), pp.data_ptr(), npart,
        0.01, err.data_ptr(), *fin, st))
    call(g1, w1, x1, y1, d1, p1, None, None, None, None)
    wout = torch.full((3, 3, 32, 32), float("nan"), device="cuda")
    dbout = torch.full((32,), float("nan"), device="cuda")
    call(g2, w2, x2, y2, d2, p2, p1.data_ptr(), d1.data_ptr(), wout.data_ptr(), dbout.data_ptr())
    call(g2, w2, x2, y2b, d2b, p2b, None, None, None, None)
    wref = torch.empty_like(wout)
    dbref = torch.empty_like(dbout)
    L.check(lib.igm_cnn_wgrad_finish(p1.data_ptr(), npart, 32, 32, wref.data_ptr(), st))
    L.check(lib.igm_reduce_partials(d1.data_ptr(), npart, 32, 32, dbref.data_ptr(), 0, st))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(wout, wref) and torch.equal(dbout, dbref)
    assert torch.equal(y2, y2b) and torch.equal(p2, p2b) and torch.equal(d2, d2b)


@pytest.mark.parametrize("B,H,W", [(1, 8, 128), (2, 9, 150), (1, 1000, 1000)])
def test_conv1x1_wgrad_is_the_centre_tap(B, H, W):
    """igm_conv1x1_wgrad: the kw = 1 partials bit for bit as igm_conv3x3_wgrad's,
    so the head's kernel gradient (igm_cnn_head_wgrad_finish) is unchanged."""
    g = torch.Generator().manual_seed(B * 3 + H + W)
    lib, st = L.lib(), L.stream_ptr()
    x = to_rc(bf(torch.randn(B, 32, H, W, generator=g))).to(torch.bfloat16).cuda()
    gd = to_rc(bf(torch.randn(B, 32, H, W, generator=g))).to(torch.bfloat16).cuda()
    npart = 148
    plen = int(lib.igm_conv3x3_wgrad_partial_len(32))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    p3 = torch.empty((npart, 3, 128, plen // 384), device="cuda")
    p1 = torch.empty_like(p3)
    L.check(lib.igm_conv3x3_wgrad(B, H, W, 32, x.data_ptr(), gd.data_ptr(), p3.data_ptr(), npart, err.data_ptr(), st))
    L.check(lib.igm_conv1x1_wgrad(B, H, W, x.data_ptr(), gd.data_ptr(), p1.data_ptr(), npart, err.data_ptr(), st))
    o3 = torch.empty((32, 20), device="cuda")
    o1 = torch.empty_like(o3)
    L.check(lib.igm_cnn_head_wgrad_finish(p3.data_ptr(), npart, 20, o3.data_ptr(), st))
    L.check(lib.igm_cnn_head_wgrad_finish(p1.data_ptr(), npart, 20, o1.data_ptr(), st))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert torch.equal(p1[:, 1], p3[:, 1])
    assert torch.equal(o1, o3)


@pytest.mark.parametrize("B,H,W,nz,mask", [(1, 4, 128, 10, False), (2, 9, 173, 10, True), (1, 1000, 1000, 10, True),
                                           (3, 5, 41, 16, True), (1, 7, 301, 5, False), (1, 1, 1, 1, True)])
def test_head_forward(B, H, W, nz, mask):
    """igm_cnn_head_forward (the 1x1 head) against a float64 evaluation of the
    same sum: FP32 fma chains over the 32 channels, so within 1e-5 of the
    output's scale; zero where thk_mask <= 0."""
    g = torch.Generator().manual_seed(B + H + W + nz)
    lib, st = L.lib(), L.stream_ptr()
    nout = 2 * nz
    a32 = bf(torch.randn(B, 32, H, W, generator=g))
    act = to_rc(a32).to(torch.bfloat16).cuda()
    wh = torch.randn(32, nout, generator=g) * 0.3
    bh = torch.randn(nout, generator=g) * 0.1
    thk = torch.rand(B, H, W, generator=g) - 0.3
    U = torch.full((B, nz, H, W), float("nan"), device="cuda")
    V = torch.full_like(U, float("nan"))
    thk_d, wh_d, bh_d = thk.cuda(), wh.cuda(), bh.cuda()  # device copies held for the call
    L.check(lib.igm_cnn_head_forward(B, H, W, nz, act.data_ptr(), wh_d.data_ptr(), bh_d.data_ptr(), 2.5,
                                     U.data_ptr(), V.data_ptr(), thk_d.data_ptr() if mask else None, st))
    torch.cuda.synchronize()
    y = (torch.einsum("bchw,cj->bjhw", a32.double(), wh.double()) + bh.double()[None, :, None, None]) * 2.5
    if mask:
        y = torch.where((thk > 0)[:, None], y, torch.zeros_like(y))
    got = torch.cat([U, V], 1).cpu().double()
    assert bool(torch.isfinite(got).all())
    assert float((got - y).abs().max()) <= 1e-5 * float(y.abs().max()) + 1e-6
    if mask:
        assert bool((got[(thk <= 0)[:, None].expand_as(got)] == 0).all())
