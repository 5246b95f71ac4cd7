"""Learned PDHG warm start: a small 3-D complex-valued convolutional encoder-decoder.

No counterpart in the reference, which always starts PDHG from zeros
(``tvme.py:190-205``, ``tvm.py:180-186``, ``tvmw.py:705-711``).  The network
maps the density-compensated adjoint image ``x0 = sum_c S_c^H F^H (w y)`` of
one (bin, echo) to an estimate of the PDHG result; PDHG then runs from that
iterate to the same stopping rule, so the returned image is still a PDHG
iterate (``solver.PdhgSolver``) and zero-start PDHG stays the fallback.

Every convolution runs in the library's BF16 tensor-core kernels with FP32
accumulation (``tr_conv3d_fwd`` for the forward pass and the data gradient,
``tr_conv3d_wgrad`` for the weight gradient); torch provides the elementwise
glue (CReLU, pooling, upsampling, loss, Adam).  Complex convolutions are real
convolutions on [re | im] channel halves with the weight structure
[[Wr, -Wi], [Wi, Wr]], so each layer is C-linear and its gradient flows to
(Wr, Wi).  Training pairs come from the b200 solver on seeded phantoms.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import asdict, dataclass
from pathlib import Path
from typing import Optional

import numpy as np

from . import _lib

WEIGHTS = Path(__file__).resolve().parent / "warmstart_net.pt"


# ---------------------------------------------------------------------- conv kernels
def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream(t):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def conv3d_fwd_bf16(x_bf, w_bf, bias=None):
    """x (N, D, H, W, Cin) bf16, w (Cout, 27, Cin) bf16 -> (N, D, H, W, Cout) f32."""
    import torch
    N, D, H, W, Cin = x_bf.shape
    Cout = w_bf.shape[0]
    y = torch.empty((N, D, H, W, Cout), dtype=torch.float32, device=x_bf.device)
    b = _ptr(bias) if bias is not None else None
    _lib.check(_lib.load().tr_conv3d_fwd(_ptr(x_bf), _ptr(w_bf), b, _ptr(y), N, D, H, W, Cin, Cout, _stream(y)),
               "tr_conv3d_fwd")
    return y


def conv3d_wgrad_bf16(x_bf, gy_bf):
    """dw (Cout, 27, Cin) f32 = sum_v gy[v, co] x[v + tap, ci]."""
    import torch
    N, D, H, W, Cin = x_bf.shape
    Cout = gy_bf.shape[-1]
    L = _lib.load()
    nbytes = ctypes.c_size_t(0)
    _lib.check(L.tr_conv3d_wgrad_workspace(N, D, H, W, Cin, Cout, ctypes.byref(nbytes)))
    ws = torch.empty(max(1, nbytes.value // 4), dtype=torch.float32, device=x_bf.device)
    dw = torch.empty((Cout, 27, Cin), dtype=torch.float32, device=x_bf.device)
    _lib.check(L.tr_conv3d_wgrad(_ptr(x_bf), _ptr(gy_bf), _ptr(dw), N, D, H, W, Cin, Cout, _ptr(ws),
                                 nbytes.value, _stream(dw)), "tr_conv3d_wgrad")
    return dw


def _flip_swap(w):
    """w (Cout, 27, Cin) -> w' (Cin, 27, Cout) with taps reversed (the data-gradient weights)."""
    return w.flip(1).permute(2, 1, 0).contiguous()


def conv3d_dgrad_bf16(gy_bf, w_bf):
    """Gradient w.r.t. the input: the forward kernel on the flipped, channel-swapped
    weights, with their output channels padded to a multiple of 8."""
    import torch
    wt = _flip_swap(w_bf)
    cin = wt.shape[0]
    pad = (-cin) % 8
    if pad:
        wt = torch.cat([wt, wt.new_zeros((pad,) + tuple(wt.shape[1:]))], dim=0)
    gx = conv3d_fwd_bf16(gy_bf, wt)
    return gx[..., :cin].contiguous() if pad else gx


def _make_conv_fn():
    import torch

    class Conv3dBF16(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x, w, b):
            xb = x.contiguous().to(torch.bfloat16)
            wb = w.contiguous().to(torch.bfloat16)
            ctx.save_for_backward(xb, wb)
            return conv3d_fwd_bf16(xb, wb, b)

        @staticmethod
        def backward(ctx, gy):
            xb, wb = ctx.saved_tensors
            gb = gy.contiguous().to(torch.bfloat16)
            gx = conv3d_dgrad_bf16(gb, wb) if ctx.needs_input_grad[0] else None
            gw = conv3d_wgrad_bf16(xb, gb) if ctx.needs_input_grad[1] else None
            gbias = gy.sum(dim=(0, 1, 2, 3)) if ctx.needs_input_grad[2] else None
            return gx, gw, gbias

    return Conv3dBF16


_CONV = None


def conv3d(x, w, b):
    global _CONV
    if _CONV is None:
        _CONV = _make_conv_fn()
    return _CONV.apply(x, w, b)


# ---------------------------------------------------------------------- network
@dataclass
class NetConfig:
    widths: tuple = (8, 16, 32)      # complex channels per level
    levels: int = 3


def _build_modules(cfg: NetConfig):
    import torch
    import torch.nn as nn

    class ComplexConv3d(nn.Module):
        """C-linear 3x3x3 convolution on channels-last [re | im] tensors."""

        def __init__(self, cin, cout):
            super().__init__()
            scale = 1.0 / math.sqrt(27 * cin * 2)
            self.cin, self.cout = cin, cout
            self.wr = nn.Parameter(torch.randn(cout, 27, cin) * scale)
            self.wi = nn.Parameter(torch.randn(cout, 27, cin) * scale)
            self.br = nn.Parameter(torch.zeros(cout))
            self.bi = nn.Parameter(torch.zeros(cout))
            self.pad = (-2 * cout) % 8        # the kernels want Cout % 8 == 0

        def forward(self, x):
            top = torch.cat([self.wr, -self.wi], dim=2)
            bot = torch.cat([self.wi, self.wr], dim=2)
            w = torch.cat([top, bot], dim=0)                    # (2 cout, 27, 2 cin)
            b = torch.cat([self.br, self.bi])
            if self.pad:
                w = torch.cat([w, w.new_zeros(self.pad, 27, 2 * self.cin)], dim=0)
                b = torch.cat([b, b.new_zeros(self.pad)])
            y = conv3d(x, w, b)
            return y[..., : 2 * self.cout] if self.pad else y

    def crelu(x):
        return torch.relu(x)

    def down(x):
        N, D, H, W, C = x.shape
        return x.view(N, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(dim=(2, 4, 6))

    def up(x):
        N, D, H, W, C = x.shape
        x = x[:, :, None, :, None, :, None, :].expand(N, D, 2, H, 2, W, 2, C)
        return x.reshape(N, 2 * D, 2 * H, 2 * W, C)

    def cat_c(a, b):
        """Concatenate complex channels of two [re | im] tensors."""
        ca, cb = a.shape[-1] // 2, b.shape[-1] // 2
        return torch.cat([a[..., :ca], b[..., :cb], a[..., ca:], b[..., cb:]], dim=-1)

    class WarmStartNet(nn.Module):
        def __init__(self, c: NetConfig):
            super().__init__()
            w = c.widths
            self.widths = tuple(w)
            self.enc = nn.ModuleList()
            cin = 1
            for i in range(c.levels):
                self.enc.append(nn.ModuleList([ComplexConv3d(cin, w[i]), ComplexConv3d(w[i], w[i])]))
                cin = w[i]
            self.dec = nn.ModuleList()
            for i in range(c.levels - 2, -1, -1):
                self.dec.append(nn.ModuleList([ComplexConv3d(w[i + 1], w[i]), ComplexConv3d(2 * w[i], w[i])]))
            self.out = ComplexConv3d(w[0], 1)
            self.skip = nn.Parameter(torch.tensor([1.0, 0.0]))   # complex gain on the input

        def forward(self, x):
            """x: (N, D, H, W, 2) channels-last [re, im]; returns the same shape."""
            skips = []
            h = x
            for i, (c1, c2) in enumerate(self.enc):
                if i > 0:
                    h = down(h)
                h = crelu(c2(crelu(c1(h))))
                skips.append(h)
            for j, (cu, cc) in enumerate(self.dec):
                h = crelu(cu(up(h)))
                h = crelu(cc(cat_c(h, skips[-2 - j])))
            d = self.out(h)
            sr, si = self.skip[0], self.skip[1]
            xr, xi = x[..., 0:1], x[..., 1:2]
            return d + torch.cat([sr * xr - si * xi, sr * xi + si * xr], dim=-1)

    return WarmStartNet


def build_net(cfg: Optional[NetConfig] = None):
    return _build_modules(cfg or NetConfig())(cfg or NetConfig())


def count_params(net) -> int:
    return int(sum(p.numel() for p in net.parameters()))


def to_channels_last(c):
    """(..., D, H, W) complex -> (N, D, H, W, 2) float32."""
    import torch
    c = c.reshape((-1,) + tuple(c.shape[-3:]))
    return torch.stack([c.real, c.imag], dim=-1).float().contiguous()


def from_channels_last(r, shape):
    import torch
    return torch.complex(r[..., 0], r[..., 1]).reshape(shape)


# ---------------------------------------------------------------------- inference
def predict(net, x0, chunk: int = 1):
    """Apply the network to every (bin, echo) image of x0 (B, E, Z, Y, X) complex64.

    Inputs are scaled by 1 / max|x0| (the network is trained scale-free) and the
    output is scaled back.  Volumes are padded to multiples of 2^(levels-1).
    """
    import torch
    shape = tuple(x0.shape)
    Z, Y, X = shape[-3:]
    m = 2 ** (len(net.enc) - 1)
    pz, py, px = (-Z) % m, (-Y) % m, (-X) % m
    scale = float(x0.abs().max())
    scale = scale if scale > 0 else 1.0
    imgs = x0.reshape((-1, Z, Y, X))
    out = torch.empty_like(imgs)
    with torch.no_grad():
        for i in range(0, imgs.shape[0], chunk):
            a = imgs[i:i + chunk] / scale
            if pz or py or px:
                a = torch.nn.functional.pad(a, (0, px, 0, py, 0, pz))
            r = net(to_channels_last(a))
            y = from_channels_last(r, a.shape)[:, :Z, :Y, :X]
            out[i:i + chunk] = y * scale
    return out.reshape(shape)


def save_model(net, path: Path = WEIGHTS, meta: Optional[dict] = None):
    import torch
    torch.save({"state_dict": {k: v.detach().cpu() for k, v in net.state_dict().items()},
                "config": asdict(NetConfig(widths=tuple(net.widths), levels=len(net.enc))),
                "meta": meta or {}}, path)


def load_model(path: Path = WEIGHTS, device="cuda"):
    """The trained network; raises FileNotFoundError when none has been trained."""
    import torch
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(f"no trained warm-start network at {path}")
    ck = torch.load(path, map_location="cpu", weights_only=False)
    cfg = NetConfig(widths=tuple(ck["config"]["widths"]), levels=int(ck["config"]["levels"]))
    net = build_net(cfg)
    net.load_state_dict(ck["state_dict"])
    net.meta = ck.get("meta", {})
    return net.to(device).eval()


def warm_solve(solver, cfg=None, max_iter: int = 300, tol: float = 1e-3, model=None):
    """Warm-started PDHG: u = u_bar = net(x0) and the data dual at its fixed-point
    relation q = A u - y; returns the solver's SolveResult with ``seconds`` covering
    the network inference, the dual set-up and the iterations (CUDA events)."""
    import torch
    net = model if model is not None else load_model(device=solver.device)
    start = torch.cuda.Event(enable_timing=True)
    mid = torch.cuda.Event(enable_timing=True)
    start.record()
    x0 = solver.adjoint_image()
    u0 = predict(net, x0)
    q0 = solver.data_residual(u0)          # data dual consistent with u0
    mid.record()
    res = solver.run(max_iter=max_iter, tol=tol, init={"u": u0, "u_bar": u0, "q": q0})
    mid.synchronize()
    res.seconds += start.elapsed_time(mid) / 1e3
    res.inference_seconds = start.elapsed_time(mid) / 1e3
    return res


# ---------------------------------------------------------------------- training
def make_pairs(n: int, base_cfg, device=0, max_iter: int = 300, tol: float = 1e-3, seed0: int = 1000,
               step_rule: str = "reference"):
    """(x0, target) volumes from n seeded phantoms: x0 the density-compensated
    adjoint, target the plain b200 PDHG result at (tol, max_iter) under
    ``step_rule``; both (n*B*E, Z, Y, X) complex64."""
    import torch
    from dataclasses import replace
    from . import synthetic as syn
    from .solver import PdhgSolver
    xs, ys = [], []
    for i in range(n):
        cfg = replace(base_cfg, seed=seed0 + i)
        ds = syn.make_geometry(cfg)
        syn.simulate_kspace_b200(ds, device)
        s = PdhgSolver(cfg.algorithm, cfg.img_shape, [ds.coord[ds.bin_indices(b)] for b in range(cfg.n_bins)],
                       ds.bin_dcf(), ds.mps, ds.bin_ksp(), l2_coupling=cfg.l2_coupling, lam_m=cfg.lam,
                       lam_e=cfg.lam, lam_w1=cfg.lam, lam_w2=cfg.lam, device=device, step_rule=step_rule)
        x0 = s.adjoint_image()
        r = s.run(max_iter=max_iter, tol=tol)
        scale = float(x0.abs().max()) or 1.0
        xs.append((x0 / scale).reshape((-1,) + tuple(cfg.img_shape)).cpu())
        ys.append((r.image / scale).reshape((-1,) + tuple(cfg.img_shape)).cpu())
        s.close()
        torch.cuda.empty_cache()
    return torch.cat(xs), torch.cat(ys)


def train(x0, target, steps: int = 400, crop=(32, 32, 32), batch: int = 4, lr: float = 2e-3,
          cfg: Optional[NetConfig] = None, device="cuda", seed: int = 0, log_every: int = 50):
    """Adam on random crops; loss = ||net(x0) - target||^2 / ||target||^2 per crop."""
    import torch
    g = torch.Generator().manual_seed(seed)
    net = build_net(cfg).to(device)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    n, Z, Y, X = x0.shape
    cz, cy, cx = crop
    history = []
    t0 = time.perf_counter()
    for it in range(steps):
        idx = torch.randint(0, n, (batch,), generator=g)
        oz = torch.randint(0, Z - cz + 1, (batch,), generator=g)
        oy = torch.randint(0, Y - cy + 1, (batch,), generator=g)
        ox = torch.randint(0, X - cx + 1, (batch,), generator=g)
        a = torch.stack([x0[idx[j], oz[j]:oz[j] + cz, oy[j]:oy[j] + cy, ox[j]:ox[j] + cx] for j in range(batch)])
        b = torch.stack([target[idx[j], oz[j]:oz[j] + cz, oy[j]:oy[j] + cy, ox[j]:ox[j] + cx] for j in range(batch)])
        a, b = a.to(device), b.to(device)
        pred = from_channels_last(net(to_channels_last(a)), a.shape)
        num = (pred - b).abs().pow(2).sum(dim=(1, 2, 3))
        den = b.abs().pow(2).sum(dim=(1, 2, 3)).clamp_min(1e-12)
        loss = (num / den).mean()
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        if it % log_every == 0 or it == steps - 1:
            history.append((it, float(loss.detach())))
    return net, {"history": history, "seconds": time.perf_counter() - t0}


def relative_error(net, x0, target, device="cuda", limit: int = 8) -> float:
    """Mean relative L2 error of the prediction on whole volumes."""
    import torch
    errs = []
    for i in range(min(limit, x0.shape[0])):
        a = x0[i:i + 1].to(device)
        p = predict(net, a[None])[0]
        t = target[i:i + 1].to(device)
        errs.append(float((p - t).norm() / t.norm().clamp_min(1e-12)))
    return float(np.mean(errs))


# ---------------------------------------------------------------------- evaluation
def holdout_eval(net, cfg, seed: int, max_iter: int = 300, tol: float = 1e-3, ref_iter: int = 0, device=0,
                 step_rule: str = "reference") -> dict:
    """Plain and warm-started solves of one unseen phantom to (tol, max_iter).

    With ref_iter > 0 a zero-start solve of ref_iter iterations (no stopping
    rule) stands in for the PDHG fixed point, and both results report their
    relative L2 distance to it."""
    from dataclasses import replace
    from . import synthetic as syn
    from .solver import PdhgSolver
    hcfg = replace(cfg, seed=seed)
    ds = syn.make_geometry(hcfg)
    syn.simulate_kspace_b200(ds, device)
    s = PdhgSolver(hcfg.algorithm, hcfg.img_shape, [ds.coord[ds.bin_indices(b)] for b in range(hcfg.n_bins)],
                   ds.bin_dcf(), ds.mps, ds.bin_ksp(), l2_coupling=hcfg.l2_coupling, lam_m=hcfg.lam,
                   lam_e=hcfg.lam, lam_w1=hcfg.lam, lam_w2=hcfg.lam, device=device, step_rule=step_rule)
    rel = lambda a, b: float((a - b).norm() / b.norm().clamp_min(1e-30))
    plain = s.run(max_iter=max_iter, tol=tol)
    plain_img = plain.image.clone()
    net.eval()
    warm = warm_solve(s, hcfg, max_iter=max_iter, tol=tol, model=net)
    out = {"workload": hcfg.name, "seed": seed, "step_rule": step_rule, "plain_iterations": plain.iterations,
           "plain_seconds": plain.seconds, "plain_final_tol": plain.tols[-1] if plain.tols else None,
           "warm_iterations": warm.iterations, "warm_seconds": warm.seconds,
           "warm_final_tol": warm.tols[-1] if warm.tols else None,
           "warm_inference_seconds": warm.inference_seconds,
           "rel_l2_warm_vs_plain": rel(warm.image, plain_img)}
    if ref_iter > 0:
        warm_img = warm.image.clone()
        ref = s.run(max_iter=ref_iter, tol=0.0)
        out["ref_iterations"] = ref.iterations
        out["rel_l2_plain_vs_ref"] = rel(plain_img, ref.image)
        out["rel_l2_warm_vs_ref"] = rel(warm_img, ref.image)
    s.close()
    return out


# ---------------------------------------------------------------------- command line
def main(argv=None):
    """Train the warm-start network on b200 PDHG solutions of seeded phantoms.

        python -m multinodemri-miccai26_b200.warmstart --phantoms 16 --steps 600 --out warmstart_net.pt
        python -m multinodemri-miccai26_b200.warmstart --eval --out warmstart_net.pt --ref-iter 1500
    """
    import argparse
    import json
    from . import synthetic as syn
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="warm-96")
    ap.add_argument("--phantoms", type=int, default=16)
    ap.add_argument("--holdout", type=int, default=2)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--crop", type=int, nargs=3, default=[32, 32, 32])
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--widths", type=int, nargs="+", default=[16, 32, 64])
    ap.add_argument("--max-iter", type=int, default=300, help="iteration cap of the evaluated solves")
    ap.add_argument("--target-iter", type=int, default=300,
                    help="iterations of the zero-start solves that make the training targets")
    ap.add_argument("--target-tol", type=float, default=None, help="stopping tolerance of the target solves")
    ap.add_argument("--ref-iter", type=int, default=0, help="iterations of the fixed-point stand-in (0: none)")
    ap.add_argument("--eval", action="store_true", help="evaluate the network at --out; no training")
    ap.add_argument("--eval-config", default=None, help="workload of the held-out solve (default --config)")
    ap.add_argument("--step-rule", choices=("reference", "power"), default="power",
                    help="PDHG steps of the target and evaluation solves")
    ap.add_argument("--out", default=str(WEIGHTS))
    args = ap.parse_args(argv)
    cfg = syn.CONFIGS[args.config]
    ecfg = syn.CONFIGS[args.eval_config or args.config]
    seed_eval = 1000 + args.phantoms + args.holdout + 7
    if args.eval:
        net = load_model(Path(args.out))
        res = holdout_eval(net, ecfg, seed_eval, max_iter=args.max_iter, tol=ecfg.tol, ref_iter=args.ref_iter,
                           step_rule=args.step_rule)
        print(json.dumps({"eval": res, "trained": {k: v for k, v in net.meta.items() if k != "loss_history"}}))
        return
    t_tol = cfg.tol if args.target_tol is None else args.target_tol
    t0 = time.perf_counter()
    x0, tgt = make_pairs(args.phantoms + args.holdout, cfg, max_iter=args.target_iter, tol=t_tol,
                         step_rule=args.step_rule)
    t_pairs = time.perf_counter() - t0
    n_train = args.phantoms * cfg.n_bins * cfg.n_echoes
    net_cfg = NetConfig(widths=tuple(args.widths), levels=len(args.widths))
    net, info = train(x0[:n_train], tgt[:n_train], steps=args.steps, crop=tuple(args.crop), batch=args.batch,
                      lr=args.lr, cfg=net_cfg)
    err_train = relative_error(net, x0[:n_train], tgt[:n_train])
    err_hold = relative_error(net, x0[n_train:], tgt[n_train:])
    base_hold = float(np.mean([float((x0[i] * (tgt[i].norm() / x0[i].norm()) - tgt[i]).norm() / tgt[i].norm())
                               for i in range(n_train, min(x0.shape[0], n_train + 8))]))
    meta = {"config": cfg.name, "phantoms": args.phantoms, "holdout": args.holdout, "steps": args.steps,
            "params": count_params(net), "pairs_seconds": t_pairs, "train_seconds": info["seconds"],
            "rel_err_train": err_train, "rel_err_holdout": err_hold, "rel_err_holdout_scaled_adjoint": base_hold,
            "loss_history": info["history"],
            "target": f"zero-start b200 PDHG, {args.step_rule} step rule, max_iter {args.target_iter}, tol {t_tol}"}
    meta["holdout_solve"] = holdout_eval(net, ecfg, seed_eval, max_iter=args.max_iter, tol=ecfg.tol,
                                         ref_iter=args.ref_iter, step_rule=args.step_rule)
    save_model(net, Path(args.out), meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
