"""Test infrastructure: a float64 PyTorch (CPU) restatement of the learned denoiser's network,
loss and gradients, used only by tests to check the tensor-core kernels.

It follows kpcn.cu's definition layer by layer: features (log1p colour, albedo, normal,
depth/(depth+3), zero-padded to 16 channels), 3x3 convolutions with zero padding, 2x2 average pooling whose mean leaves out children beyond an odd edge,
nearest 2x upsampling cropped to the skip tensor's size, [upsampled, skip] concatenation, a 1x1 output convolution whose channels
[25s, 25s + 25) are softmax-normalised into the 5x5 filter of stage s, the three stages applied
in turn at dilations 1, 2, 4 with clamp-to-edge neighbours, starting from the noisy colour, and
the relative L2 loss sum((f - t)^2 / (t^2 + 0.01)) / (3 pixels).  Parameters use the flat
layout of wgpt_kpcn_get_params (per layer W[cout][ky*3+kx][cin], then bias).  Inputs and
weights can be rounded to bfloat16 first, as the GPU stores them.  With `bf16_activations` the
restatement also rounds where the GPU kernels store bfloat16 tensors: every post-ReLU layer
output and every pooled tensor on the way forward, and the gradient flowing back into each of
them; the output logits are kept in FP32 and their gradient is rounded to bfloat16 (the
filter's backward pass stores it so).  Everything between those points stays float64.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from webgpuraytracer_b200.kpcn import LAYERS, param_slices


def bf16_round(a: np.ndarray) -> np.ndarray:
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return (((u + r) >> 16) << 16).astype(np.uint32).view(np.float32)


def _bf16_t(x: torch.Tensor) -> torch.Tensor:
    """Round a float64 tensor to bfloat16 values (through float32, nearest even)."""
    return torch.from_numpy(bf16_round(x.detach().numpy().astype(np.float32)).astype(np.float64))


class _RoundBF16(torch.autograd.Function):
    """Forward and backward values rounded to bfloat16, as stored by the GPU kernels."""

    @staticmethod
    def forward(ctx, x):
        return _bf16_t(x)

    @staticmethod
    def backward(ctx, g):
        return _bf16_t(g)


class _RoundLogits(torch.autograd.Function):
    """FP32 logits forward; bfloat16 logit gradients backward."""

    @staticmethod
    def forward(ctx, x):
        return torch.from_numpy(x.detach().numpy().astype(np.float32).astype(np.float64))

    @staticmethod
    def backward(ctx, g):
        return _bf16_t(g)


def features(noisy: np.ndarray, gbuf: np.ndarray) -> np.ndarray:
    """(H, W, 16) input features from an rgba32f accumulation and a 12-float G-buffer."""
    h, w = noisy.shape[:2]
    f = np.zeros((h, w, 16), np.float32)
    f[..., 0:3] = np.log1p(np.maximum(noisy[..., :3], 0.0))
    f[..., 3:6] = gbuf[..., 4:7]
    f[..., 6:9] = gbuf[..., 0:3]
    d = np.maximum(gbuf[..., 11], 0.0)
    f[..., 9] = d / (d + 3.0)
    return f


def unpack(params: np.ndarray, round_bf16: bool):
    """Per layer (torch weight [cout, cin, k, k] float64, bias [cout] float64)."""
    sl = param_slices()
    out = {}
    for l in LAYERS:
        ws, bs = sl[l.name]
        w = params[ws].astype(np.float32)
        if round_bf16:
            w = bf16_round(w)
        k = 3 if l.taps == 9 else 1
        w = w.reshape(l.cout, k, k, l.cin).transpose(0, 3, 1, 2)
        out[l.name] = (torch.tensor(np.ascontiguousarray(w), dtype=torch.float64, requires_grad=True),
                       torch.tensor(params[bs].astype(np.float64), requires_grad=True))
    return out


def forward_loss(params: np.ndarray, noisy: np.ndarray, gbuf: np.ndarray, target: np.ndarray,
                 round_bf16: bool = True, bf16_activations: bool = False):
    """Returns (loss tensor, filtered (H, W, 3) tensor, per-layer parameter tensors)."""
    q = _RoundBF16.apply if bf16_activations else (lambda a: a)
    x = features(noisy, gbuf)
    if round_bf16:
        x = bf16_round(x)
    P = unpack(params, round_bf16)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64)
    X = t(x).permute(2, 0, 1)[None]

    def conv(name, inp, relu=True):
        w, b = P[name]
        pad = 1 if w.shape[-1] == 3 else 0
        y = F.conv2d(inp, w, b, padding=pad)
        return q(F.relu(y)) if relu else y

    def pool(a):
        return q(F.avg_pool2d(a, 2, 2, ceil_mode=True, count_include_pad=False))

    def up(a, like):
        return F.interpolate(a, scale_factor=2, mode="nearest")[..., :like.shape[-2], :like.shape[-1]]

    e0 = conv("E0", conv("E0a", X))
    e1 = conv("E1", pool(e0))
    e2 = conv("E2", pool(e1))
    e3 = conv("E3", pool(e2))
    e4 = conv("E4", conv("E4a", pool(e3)))
    d3 = conv("D3", torch.cat([up(e4, e3), e3], 1))
    d2 = conv("D2", torch.cat([up(d3, e2), e2], 1))
    d1 = conv("D1", torch.cat([up(d2, e1), e1], 1))
    d0 = conv("D0", torch.cat([up(d1, e0), e0], 1))
    logits = conv("OUT", d0, relu=False)
    if bf16_activations:
        logits = _RoundLogits.apply(logits)
    logits = logits[0]                                         # (80, H, W)
    h, w = noisy.shape[:2]
    f = t(noisy[..., :3]).permute(2, 0, 1)                     # (3, H, W)
    for stage, d in enumerate((1, 2, 4)):
        wk = torch.softmax(logits[25 * stage:25 * stage + 25], 0)
        fp = F.pad(f[None], (2 * d, 2 * d, 2 * d, 2 * d), mode="replicate")[0]
        g = torch.zeros(3, h, w, dtype=torch.float64)
        for k in range(25):
            oy, ox = 2 * d + d * (k // 5 - 2), 2 * d + d * (k % 5 - 2)
            g = g + wk[k][None] * fp[:, oy:oy + h, ox:ox + w]
        f = g
    tg = t(target[..., :3]).permute(2, 0, 1)
    loss = ((f - tg) ** 2 / (tg ** 2 + 0.01)).sum() / (3.0 * h * w)
    return loss, f.permute(1, 2, 0), P


def loss_and_grads(params: np.ndarray, noisy, gbuf, target, round_bf16: bool = True,
                   bf16_activations: bool = False):
    """(loss, flat gradient in the wgpt_kpcn layout, filtered (H, W, 3)) in float64."""
    loss, f, P = forward_loss(params, noisy, gbuf, target, round_bf16, bf16_activations)
    loss.backward()
    g = np.zeros(params.size, np.float64)
    sl = param_slices()
    for l in LAYERS:
        w, b = P[l.name]
        ws, bs = sl[l.name]
        g[ws] = w.grad.numpy().transpose(0, 2, 3, 1).reshape(-1)
        g[bs] = b.grad.numpy()
    return float(loss.item()), g, f.detach().numpy()
