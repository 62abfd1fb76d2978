"""Learned warm start: the BF16 tensor-core 3x3x3 convolutions against PyTorch's FP32
convolution on the CPU (forward, data gradient, weight gradient), and a small end-to-end run
(data from the library's own projector, noise and CGLS; U-Net training; warm-started CGLS)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf16_round(a):
    import torch
    return torch.from_numpy(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).float()


def _ref_weights(w, cin, cout):
    """(Cout, 27*Cin) with tap (dz*3+dy)*3+dx major -> (Cout, Cin, 3, 3, 3) for F.conv3d."""
    return w.view(cout, 27, cin).permute(0, 2, 1).reshape(cout, cin, 3, 3, 3)


@pytest.mark.parametrize("shape,cin,cout", [((6, 5, 7), 3, 5), ((20, 16, 16), 40, 70), ((8, 8, 8), 1, 16),
                                            ((4, 9, 6), 48, 1),
                                            # tcgen05 path: Cin % 8 == 0 and Cout % 16 == 0, N tiles 16..128
                                            ((8, 6, 10), 16, 16), ((7, 9, 11), 8, 32), ((9, 8, 7), 48, 48),
                                            ((6, 6, 6), 24, 64), ((5, 7, 9), 16, 128), ((3, 4, 5), 64, 192),
                                            # halo-tile kernel: Cin % 16 == 0, W % 8 == 0, H % 16 == 0
                                            ((4, 16, 8), 16, 16), ((8, 32, 16), 32, 32), ((6, 16, 24), 48, 16),
                                            ((4, 16, 8), 16, 64), ((2, 16, 8), 64, 128), ((2, 16, 16), 32, 192),
                                            ((5, 16, 8), 96, 32)])
@pytest.mark.parametrize("tcgen05", [0, 1, 3])
def test_conv3d_matches_torch_fp32(shape, cin, cout, tcgen05):
    import torch
    import torch.nn.functional as F
    from tigre_b200 import _native as N
    D, H, W = shape
    rng = np.random.default_rng(cin * 7 + cout)
    x = _bf16_round(rng.standard_normal((D, H, W, cin)))
    w = _bf16_round(rng.standard_normal((cout, 27 * cin)) / np.sqrt(27 * cin))
    b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32))
    dy = _bf16_round(rng.standard_normal((D, H, W, cout)))
    # CPU FP32 reference
    xr = x.permute(3, 0, 1, 2).unsqueeze(0).clone().requires_grad_(True)
    wr = _ref_weights(w, cin, cout).clone().requires_grad_(True)
    yr = F.conv3d(xr, wr, b, padding=1)
    yr.backward(dy.permute(3, 0, 1, 2).unsqueeze(0))
    y_ref = yr.detach()[0].permute(1, 2, 3, 0).numpy()
    dx_ref = xr.grad[0].permute(1, 2, 3, 0).numpy()
    dw_ref = wr.grad.permute(0, 2, 3, 4, 1).reshape(cout, 27 * cin).numpy()
    # device
    L = N.lib()
    xd = x.to(torch.bfloat16).cuda()
    wd = w.to(torch.bfloat16).cuda()
    bd = b.cuda()
    dyd = dy.to(torch.bfloat16).cuda()
    col = torch.empty(int(L.tigre_conv3d_col_elems(D, H, W, cin)), dtype=torch.bfloat16, device="cuda")
    dcol = torch.empty(int(L.tigre_conv3d_col_elems(D, H, W, cin)), dtype=torch.float32, device="cuda")
    y = torch.empty((D, H, W, cout), dtype=torch.float32, device="cuda")
    dx = torch.empty((D, H, W, cin), dtype=torch.float32, device="cuda")
    dw = torch.zeros((cout, 27 * cin), dtype=torch.float32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    old = L.tigre_conv3d_set_tcgen05(tcgen05)
    try:
        N.check(L.tigre_conv3d_fwd(p(xd), p(wd), p(bd), None, p(y), D, H, W, cin, cout, 0, p(col), None), "fwd")
    finally:
        L.tigre_conv3d_set_tcgen05(old)
    N.check(L.tigre_conv3d_bwd_data(p(dyd), p(wd), p(dx), D, H, W, cin, cout, p(dcol), None), "data")
    N.check(L.tigre_conv3d_bwd_weight(p(xd), p(dyd), p(dw), D, H, W, cin, cout, p(col), None), "weight")
    torch.cuda.synchronize()
    assert L.tigre_conv3d_status(1) == 0
    for got, ref, name in ((y, y_ref, "y"), (dx, dx_ref, "dx"), (dw, dw_ref, "dw")):
        got = got.cpu().numpy()
        # same BF16 operands, FP32 sums in another order (tensor-core accumulation): 2e-4 of the max
        err = np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30)
        assert err <= 2e-4, (name, err)


def test_conv3d_weight_gradient_is_deterministic():
    """The weight gradient sums its voxel splits in a fixed order: repeated calls give the same
    bits."""
    import torch
    from tigre_b200 import _native as N
    L = N.lib()
    D, H, W, cin, cout = 16, 32, 32, 16, 16
    g = torch.Generator("cuda").manual_seed(5)
    x = torch.randn((D, H, W, cin), device="cuda", generator=g).to(torch.bfloat16)
    dy = torch.randn((D, H, W, cout), device="cuda", generator=g).to(torch.bfloat16)
    col = torch.empty(int(L.tigre_conv3d_col_elems(D, H, W, cin)), dtype=torch.bfloat16, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    out = []
    for _ in range(3):
        dw = torch.zeros((cout, 27 * cin), dtype=torch.float32, device="cuda")
        N.check(L.tigre_conv3d_bwd_weight(p(x), p(dy), p(dw), D, H, W, cin, cout, p(col), None), "weight")
        out.append(dw.cpu())
    assert torch.equal(out[0], out[1]) and torch.equal(out[0], out[2])


def test_conv_autograd_matches_torch_fp32():
    """The autograd Function (implicit-GEMM forward, flipped-weight data gradient, im2col weight
    gradient) against F.conv3d on the CPU, with Cin and Cout multiples of 8 and not."""
    import torch
    import torch.nn.functional as F
    from tigre_b200 import warmstart as WS
    for (D, H, W), cin, cout in [((8, 6, 10), 16, 24), ((5, 7, 6), 8, 1), ((4, 4, 4), 1, 8)]:
        rng = np.random.default_rng(cin + cout)
        x = _bf16_round(rng.standard_normal((D, H, W, cin)))
        w = _bf16_round(rng.standard_normal((cout, 27 * cin)) / np.sqrt(27 * cin))
        b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32))
        dy = _bf16_round(rng.standard_normal((D, H, W, cout)))
        xd = x.to(torch.bfloat16).cuda().requires_grad_(True)
        wd = w.cuda().requires_grad_(True)
        bd = b.cuda().requires_grad_(True)
        y = WS.conv3d(xd, wd, bd, False)
        y.backward(dy.to(torch.bfloat16).cuda())
        xr = x.permute(3, 0, 1, 2).unsqueeze(0).clone().requires_grad_(True)
        wr = _ref_weights(w, cin, cout).clone().requires_grad_(True)
        br = b.clone().requires_grad_(True)
        yr = F.conv3d(xr, wr, br, padding=1)
        yr.backward(dy.permute(3, 0, 1, 2).unsqueeze(0))
        pairs = [(y.float().cpu(), yr.detach()[0].permute(1, 2, 3, 0), 1e-2),            # BF16 output
                 (xd.grad.float().cpu(), xr.grad[0].permute(1, 2, 3, 0), 1e-2),        # BF16 gradient
                 (wd.grad.cpu(), wr.grad.permute(0, 2, 3, 4, 1).reshape(cout, 27 * cin), 2e-4),
                 (bd.grad.cpu(), br.grad, 1e-5)]
        for got, ref, tol in pairs:
            err = float((got - ref).abs().max() / ref.abs().max().clamp_min(1e-30))
            assert err <= tol, ((D, H, W), cin, cout, err, tol)


def test_conv3d_relu_bias_and_bf16_output():
    import torch
    from tigre_b200 import warmstart as WS
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.standard_normal((8, 8, 8, 4)).astype(np.float32)).to(torch.bfloat16).cuda()
    w = torch.from_numpy((rng.standard_normal((6, 108)) / 10).astype(np.float32)).cuda()
    b = torch.from_numpy(rng.standard_normal(6).astype(np.float32)).cuda()
    y = WS.conv3d(x, w, b, True)
    y0 = WS.conv3d(x, w, b, False)
    assert y.dtype == torch.bfloat16 and (y >= 0).all()
    assert torch.equal(y, torch.clamp(y0, min=0))


def test_warmstart_end_to_end_small():
    """32^3: training lowers the loss, the warm start is a valid CGLS start and reaches the
    residual target; timings are reported, not asserted."""
    import torch
    from tigre_b200 import warmstart as WS
    model = WS.unet(base=8, levels=3)
    tr = WS.train(model, n_train=6, steps=40, n=32, crop=0, lr=2e-3)
    assert tr["loss_last"] < tr["loss_first"]
    ev = WS.evaluate(model, n_eval=2, n=32)
    for row in ev["cases"]:
        assert row["plain_zero"]["reached"] and row["warm"]["reached"]
    assert np.isfinite(ev["warm_over_plain_zero"])
    del torch


def test_warmstart_unrolled_cgls_training_small():
    """32^3: the data term through unrolled CGLS iterations (noiseless pairs) trains: the loss
    falls, and every gradient reaches the network through the projector pair's autograd
    Functions."""
    from tigre_b200 import warmstart as WS
    model = WS.unet(base=8, levels=3)
    tr = WS.train(model, n_train=4, steps=40, n=32, crop=0, lr=2e-3, physics=1e4, unroll=3, clean_frac=1.0,
                  img_weight=0.1)
    assert np.isfinite(tr["loss_last"]) and tr["loss_last"] < tr["loss_first"], tr
    assert all(p.grad is not None and bool(p.grad.abs().sum() > 0) for p in model.parameters())


def test_unet_glue_kernels_match_torch():
    """pool2 / up_concat / conv_in / conv_out of the fused inference pass against the same
    operations in PyTorch (FP32 reference on the same BF16 values)."""
    import torch
    import torch.nn.functional as F
    from tigre_b200 import _native as N
    L = N.lib()
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    g = torch.Generator("cuda").manual_seed(7)
    x = torch.randn((8, 12, 16, 24), device="cuda", generator=g).to(torch.bfloat16)
    y = torch.empty((4, 6, 8, 24), dtype=torch.bfloat16, device="cuda")
    N.check(L.tigre_unet_pool2(p(x), p(y), 8, 12, 16, 24, None), "pool2")
    ref = x.float().view(4, 2, 6, 2, 8, 2, 24).mean(dim=(1, 3, 5))
    assert float((y.float() - ref).abs().max()) <= float(ref.abs().max()) * 2 ** -7
    skip = torch.randn((8, 12, 16, 16), device="cuda", generator=g).to(torch.bfloat16)
    cat = torch.empty((8, 12, 16, 40), dtype=torch.bfloat16, device="cuda")
    N.check(L.tigre_unet_up_concat(p(y), 24, p(skip), 16, p(cat), 8, 12, 16, None), "up_concat")
    up = y.repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2)
    assert torch.equal(cat, torch.cat([up, skip], dim=-1))
    vol = torch.randn((8, 12, 16), device="cuda", generator=g)
    w = (torch.randn((16, 27), device="cuda", generator=g) / 5).to(torch.bfloat16)
    b = torch.randn(16, device="cuda", generator=g)
    h = torch.empty((8, 12, 16, 16), dtype=torch.bfloat16, device="cuda")
    N.check(L.tigre_unet_conv_in(p(vol), p(w), p(b), p(h), 8, 12, 16, 16, 1, None), "conv_in")
    xr = vol.to(torch.bfloat16).float()[None, None]
    ref = F.relu(F.conv3d(xr, w.float().view(16, 1, 3, 3, 3), b, padding=1))[0].permute(1, 2, 3, 0)
    assert float((h.float() - ref).abs().max()) <= float(ref.abs().max()) * 2 ** -7
    wo = (torch.randn((1, 27 * 16), device="cuda", generator=g) / 20).to(torch.bfloat16)
    out = torch.empty_like(vol)
    N.check(L.tigre_unet_conv_out(p(h), 16, p(wo), 0.25, p(vol), p(out), 8, 12, 16, None), "conv_out")
    wr = wo.float().view(1, 27, 16).permute(0, 2, 1).reshape(1, 16, 3, 3, 3)
    conv = F.conv3d(h.float().permute(3, 0, 1, 2)[None], wr, torch.tensor([0.25], device="cuda"), padding=1)[0, 0]
    ref = vol + conv.to(torch.bfloat16).float()
    assert float((out - ref).abs().max()) <= float(conv.abs().max()) * 2 ** -7


def _unet_fp32_reference(model, vol):
    """The same network in FP32 (torch conv3d on BF16-rounded weights, FP32 activations)."""
    import torch
    import torch.nn.functional as F

    def conv(x, layer):
        cout, k = layer.w.shape
        cin = k // 27
        w = layer.w.detach().to(torch.bfloat16).float().view(cout, 27, cin).permute(0, 2, 1).reshape(cout, cin, 3, 3, 3)
        y = F.conv3d(x, w, layer.b.detach(), padding=1)
        return F.relu(y) if layer.relu else y

    x = vol.to(torch.bfloat16).float()[None, None]
    skips = []
    for i, (c1, c2) in enumerate(model.enc):
        x = conv(conv(x, c1), c2)
        if i < len(model.enc) - 1:
            skips.append(x)
            x = F.avg_pool3d(x, 2)
    for (c1, c2), s in zip(model.dec, reversed(skips)):
        x = torch.cat([F.interpolate(x, scale_factor=2, mode="nearest"), s], dim=1)
        x = conv(conv(x, c1), c2)
    return vol + conv(x, model.head)[0, 0]


def test_unet_fused_inference_matches_autograd_forward():
    """UNet3D.infer (fused kernels) and the autograd forward pass on the same weights, both
    against the network in FP32: BF16 activations put each within a few 1e-2 (L2) of it, and
    the fused pass is no further from it than the autograd one (within 25 %)."""
    import torch
    from tigre_b200 import warmstart as WS
    model = WS.unet(seed=3)
    vol = torch.rand((64, 64, 64), device="cuda", generator=torch.Generator("cuda").manual_seed(4))
    with torch.no_grad():
        fused = model(vol)
        ref = _unet_fp32_reference(model, vol)
    with torch.enable_grad():
        plain = model(vol).detach()
    r = ref - vol

    def err(a):
        d = a - vol - r
        return float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(r))

    e_f, e_p = err(fused), err(plain)
    print("U-Net vs FP32 network (L2): fused %.3e, autograd %.3e" % (e_f, e_p))
    assert e_f <= 5e-2 and e_p <= 5e-2 and e_f <= 1.25 * e_p + 1e-3, (e_f, e_p)


def test_pretrained_warm_start_saves_cgls_iterations():
    """The committed U-Net (trained on the warm-start configuration: 256^3, 512^2 detector at
    0.8 mm, 90 views, I0 = 5e4) on an unseen phantom of that configuration: CGLS started from its
    output reaches the residual target in at most 60 % of the iterations from zero, with noisy
    data (target: 100 zero-start iterations + 0.1 %) and noiseless data (target 5e-3)."""
    import torch
    from tigre_b200 import warmstart as WS
    model = WS.pretrained_c5()
    assert model is not None
    for target in (None, 5e-3):
        ev = WS.evaluate(model, n_eval=1, n=256, noiseless_target=target)
        row = ev["cases"][0]
        print("target %s: zero %d, FDK %d, warm %d iterations" % (
            target, row["plain_zero"]["iters"], row["plain_fdk"]["iters"], row["warm"]["iters"]))
        assert row["warm"]["reached"] and row["warm"]["iters"] <= 0.6 * row["plain_zero"]["iters"], row
    del torch
