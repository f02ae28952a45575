"""CPU oracle of the learned denoiser (test infrastructure only).

A plain PyTorch fp32 restatement of the U-Net that libwrk's tensor-core kernels
run (offlinerenderer_b200/csrc/denoiser.cu): same layers, same parameter layout
(per layer W [Cout][3][3][Cin] then bias [Cout], layers e0a e0b e1a e1b e2a e2b
e3a e3b d2a d2b d1a d1b d0a d0b head), same input packing (log1p radiance,
albedo, normal, zero-padded to 16 channels), same residual output and L1 loss in
log space.  Values are rounded to bf16 where the GPU stores them in bf16 (input,
weights, every activation), so the forward pass matches the device up to the
order of f32 accumulation; gradients come from autograd through that graph
(straight-through rounding).

The network replaces libWR's OptiX AI denoiser
(libWR/src/internal/denoiser.cpp:17-195), which is closed code with no CPU
counterpart, so this oracle checks the kernels against the network's own
definition rather than against the reference's denoiser.  Only tests/ may
import it.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

LAYERS = [(16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128), (128, 256), (256, 256),
          (384, 128), (128, 128), (192, 64), (64, 64), (96, 32), (32, 32), (32, 3)]


class _RoundBF16(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return x.to(torch.bfloat16).to(torch.float32)

    @staticmethod
    def backward(ctx, g):
        return g


def bf(x):
    return _RoundBF16.apply(x)


def split_params(flat: np.ndarray):
    """Flat f32 parameter array -> list of (W (Cout,Cin,3,3) torch, b (Cout,) torch)."""
    out, o = [], 0
    for cin, cout in LAYERS:
        n = cout * 9 * cin
        w = torch.tensor(np.asarray(flat[o:o + n], np.float32).reshape(cout, 3, 3, cin)).permute(0, 3, 1, 2).contiguous()
        o += n
        b = torch.tensor(np.asarray(flat[o:o + cout], np.float32))
        o += cout
        out.append((w, b))
    assert o == len(flat)
    return out


def flat_grads(params) -> np.ndarray:
    parts = []
    for w, b in params:
        parts.append(w.grad.permute(0, 2, 3, 1).reshape(-1).numpy())
        parts.append(b.grad.numpy())
    return np.concatenate(parts).astype(np.float32)


def pack(rgb, albedo, normal):
    """(B,H,W,3) arrays -> (B,16,H,W) bf16-rounded input."""
    B, H, W, _ = rgb.shape
    x = torch.zeros(B, 16, H, W)
    x[:, 0:3] = torch.log1p(torch.clamp(torch.tensor(rgb), min=0)).permute(0, 3, 1, 2)
    if albedo is not None:
        x[:, 3:6] = torch.tensor(albedo).permute(0, 3, 1, 2)
    if normal is not None:
        x[:, 6:9] = torch.tensor(normal).permute(0, 3, 1, 2)
    return bf(x)


def forward(params, x):
    """Returns the head output (B,3,H,W) f32."""
    def conv(i, t, relu=True):
        w, b = params[i]
        y = F.conv2d(t, bf(w), padding=1) + b.view(1, -1, 1, 1)
        return bf(F.relu(y)) if relu else y

    def pool(t):
        return bf(F.avg_pool2d(t, 2))

    def up(t):
        return F.interpolate(t, scale_factor=2, mode="nearest")

    a0 = conv(0, x)
    s0 = conv(1, a0)
    a1 = conv(2, pool(s0))
    s1 = conv(3, a1)
    a2 = conv(4, pool(s1))
    s2 = conv(5, a2)
    a3 = conv(6, pool(s2))
    b3 = conv(7, a3)
    a4 = conv(8, torch.cat([up(b3), s2], 1))
    dec2 = conv(9, a4)
    a5 = conv(10, torch.cat([up(dec2), s1], 1))
    dec1 = conv(11, a5)
    a6 = conv(12, torch.cat([up(dec1), s0], 1))
    dec0 = conv(13, a6)
    return conv(14, dec0, relu=False)


def loss_and_grads(flat: np.ndarray, rgb, albedo, normal, target):
    """(loss, flat gradient) of the mean L1 loss in log space."""
    params = split_params(flat)
    for w, b in params:
        w.requires_grad_(True)
        b.requires_grad_(True)
    x = pack(rgb, albedo, normal)
    head = forward(params, x)
    pred = torch.log1p(torch.clamp(torch.tensor(rgb), min=0)).permute(0, 3, 1, 2) + head
    tgt = torch.log1p(torch.clamp(torch.tensor(target), min=0)).permute(0, 3, 1, 2)
    loss = (pred - tgt).abs().mean()
    loss.backward()
    return float(loss.detach()), flat_grads(params)


def denoise(flat: np.ndarray, rgb, albedo, normal) -> np.ndarray:
    """Denoised (B,H,W,3) radiance; H, W multiples of 8 (no padding here)."""
    with torch.no_grad():
        params = split_params(flat)
        x = pack(rgb, albedo, normal)
        head = forward(params, x)
        pred = torch.log1p(torch.clamp(torch.tensor(rgb), min=0)).permute(0, 3, 1, 2) + head
        return torch.clamp(torch.expm1(pred), min=0).permute(0, 2, 3, 1).numpy()
