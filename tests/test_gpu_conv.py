"""Warm-start conv kernels (BF16 tensor cores, FP32 accumulation) against the float64 CPU oracle."""

import numpy as np
import pytest

from _fixtures import pkg
from oracle import conv as oconv

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _bf16_round(a):
    import torch
    return torch.from_numpy(np.asarray(a, np.float32)).bfloat16().float().numpy()


@pytest.mark.parametrize("shape,cin,cout", [((2, 6, 5, 7), 2, 8), ((1, 5, 6, 4), 16, 16), ((2, 4, 4, 4), 24, 40),
                                            ((1, 8, 8, 8), 64, 128), ((1, 9, 7, 5), 34, 24)])
def test_conv_forward_and_gradients(shape, cin, cout):
    torch = _torch()
    ws = pkg("warmstart")
    rng = np.random.default_rng(cin * 7 + cout)
    x = _bf16_round(rng.standard_normal(shape + (cin,)))
    w = _bf16_round(rng.standard_normal((cout, 27, cin)) * 0.2)
    b = rng.standard_normal(cout).astype(np.float32)
    gy = _bf16_round(rng.standard_normal(shape + (cout,)))
    xb = torch.from_numpy(x).cuda().bfloat16()
    wb = torch.from_numpy(w).cuda().bfloat16()
    y = ws.conv3d_fwd_bf16(xb, wb, torch.from_numpy(b).cuda()).cpu().numpy()
    yr = oconv.conv3d(x, w, b)
    assert np.abs(y - yr).max() <= 1e-4 * np.abs(yr).max()
    dw = ws.conv3d_wgrad_bf16(xb, torch.from_numpy(gy).cuda().bfloat16()).cpu().numpy()
    dwr = oconv.conv3d_wgrad(x, gy)
    assert np.abs(dw - dwr).max() <= 1e-4 * np.abs(dwr).max()
    # data gradient = forward with flipped, channel-swapped weights
    dx = ws.conv3d_dgrad_bf16(torch.from_numpy(gy).cuda().bfloat16(), wb).cpu().numpy()
    dxr = oconv.conv3d_dgrad(gy, w)
    assert np.abs(dx - dxr).max() <= 1e-4 * np.abs(dxr).max()


def test_wgrad_is_deterministic():
    torch = _torch()
    ws = pkg("warmstart")
    x = torch.randn(2, 16, 16, 16, 32, device="cuda").bfloat16()
    g = torch.randn(2, 16, 16, 16, 64, device="cuda").bfloat16()
    a = ws.conv3d_wgrad_bf16(x, g)
    assert torch.equal(a, ws.conv3d_wgrad_bf16(x, g))


def _network_grads(round_bf16):
    """Loss and gradients of the complex encoder-decoder: GPU kernels and a float64
    CPU oracle (optionally rounding conv operands to bf16 where the GPU path does)."""
    import torch
    import torch.autograd as ag
    ws = pkg("warmstart")
    torch.manual_seed(0)
    cfg = ws.NetConfig(widths=(4, 8, 8), levels=3)
    net = ws.build_net(cfg).cuda()
    with torch.no_grad():
        for p in net.parameters():                 # bf16-representable weights
            p.copy_(p.bfloat16().float())
    x = (torch.randn(1, 8, 8, 8, 2) * 0.5).bfloat16().float()
    t = torch.randn(1, 8, 8, 8, 2)
    loss = ((net(x.cuda()) - t.cuda()) ** 2).sum()
    loss.backward()
    g_gpu = {n: p.grad.detach().cpu().double() for n, p in net.named_parameters()}
    rnd = (lambda a: a.bfloat16().double()) if round_bf16 else (lambda a: a)

    class OracleConv(ag.Function):
        @staticmethod
        def forward(ctx, xx, w, b):
            xx, w = rnd(xx), rnd(w)
            ctx.save_for_backward(xx, w)
            return torch.from_numpy(oconv.conv3d(xx.numpy(), w.numpy(), b.numpy()))

        @staticmethod
        def backward(ctx, gy):
            xx, w = ctx.saved_tensors
            g = rnd(gy)
            return (torch.from_numpy(oconv.conv3d_dgrad(g.numpy(), w.numpy())),
                    torch.from_numpy(oconv.conv3d_wgrad(xx.numpy(), g.numpy())), gy.sum(dim=(0, 1, 2, 3)))

    saved = ws.conv3d
    try:
        ws.conv3d = lambda a, w, b: OracleConv.apply(a.double(), w.double(), b.double())
        cpu = ws.build_net(cfg).double()
        cpu.load_state_dict({k: v.detach().cpu().double() for k, v in net.state_dict().items()})
        loss_c = ((cpu(x.double()) - t.double()) ** 2).sum()
        loss_c.backward()
    finally:
        ws.conv3d = saved
    g_cpu = {n: p.grad.detach() for n, p in cpu.named_parameters()}
    return float(loss.detach()), float(loss_c.detach()), g_gpu, g_cpu


def _compare(g_gpu, g_cpu):
    import torch
    worst_cos, worst_rel = 1.0, 0.0
    for n, r in g_cpu.items():
        a, r = g_gpu[n].flatten(), r.flatten()
        worst_cos = min(worst_cos, float(torch.dot(a, r) / (a.norm() * r.norm() + 1e-30)))
        worst_rel = max(worst_rel, float((a - r).norm() / (r.norm() + 1e-30)))
    return worst_cos, worst_rel


def test_network_gradients_match_cpu_oracle():
    """The kernels: with operands rounded to bf16 at the same points, GPU (FP32 accumulation)
    and CPU (float64) loss gradients of the whole network agree to accumulation error."""
    _torch()
    l_g, l_c, g_gpu, g_cpu = _network_grads(round_bf16=True)
    assert abs(l_g - l_c) <= 1e-4 * abs(l_c)
    cos, rel = _compare(g_gpu, g_cpu)
    assert cos > 0.9999 and rel < 1e-2, (cos, rel)


def test_network_gradients_bf16_precision_bound():
    """Against an all-float64 oracle the BF16 path stays within the expected precision."""
    _torch()
    l_g, l_c, g_gpu, g_cpu = _network_grads(round_bf16=False)
    assert abs(l_g - l_c) <= 3e-2 * abs(l_c)
    cos, rel = _compare(g_gpu, g_cpu)
    assert cos > 0.95 and rel < 0.35, (cos, rel)


def test_training_reduces_loss():
    torch = _torch()
    ws = pkg("warmstart")
    torch.manual_seed(0)
    x0 = torch.randn(3, 16, 16, 16, dtype=torch.complex64)
    target = 0.5 * x0 + 0.1 * torch.roll(x0, 1, dims=-1)
    net, info = ws.train(x0, target, steps=60, crop=(16, 16, 16), batch=2, cfg=ws.NetConfig(widths=(4, 8, 8)),
                         log_every=10)
    h = info["history"]
    assert h[-1][1] < 0.5 * h[0][1]
    err = ws.relative_error(net, x0, target)
    assert err < 0.8
