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


def test_network_gradients_match_cpu_oracle():
    """Loss gradients of the whole complex encoder-decoder, GPU kernels vs float64 CPU convolutions."""
    torch = _torch()
    ws = pkg("warmstart")
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
    # CPU oracle: the same module graph with its convolutions swapped for the float64 NumPy conv
    import torch.autograd as ag

    class OracleConv(ag.Function):
        @staticmethod
        def forward(ctx, xx, w, b):
            ctx.save_for_backward(xx, w)
            return torch.from_numpy(oconv.conv3d(xx.numpy(), w.numpy(), b.numpy()))

        @staticmethod
        def backward(ctx, gy):
            xx, w = ctx.saved_tensors
            return (torch.from_numpy(oconv.conv3d_dgrad(gy.numpy(), w.numpy())),
                    torch.from_numpy(oconv.conv3d_wgrad(xx.numpy(), gy.numpy())), gy.sum(dim=(0, 1, 2, 3)))

    saved = ws.conv3d
    try:
        ws.conv3d = lambda a, w, b: OracleConv.apply(a.double(), w.double(), b.double())
        cpu = ws.build_net(cfg).double()
        cpu.load_state_dict({k: v.detach().cpu().double() for k, v in net.state_dict().items()})
        loss_c = ((cpu(x.double()) - t.double()) ** 2).sum()
        loss_c.backward()
    finally:
        ws.conv3d = saved
    assert abs(float(loss.detach()) - float(loss_c.detach())) <= 2e-2 * abs(float(loss_c.detach()))
    for n, p in cpu.named_parameters():
        a, r = g_gpu[n].flatten(), p.grad.flatten()
        cos = float(torch.dot(a, r) / (a.norm() * r.norm() + 1e-30))
        assert cos > 0.995, (n, cos)
        assert float((a - r).norm() / (r.norm() + 1e-30)) < 0.1, n


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
