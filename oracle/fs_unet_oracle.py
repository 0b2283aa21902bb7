"""CPU FP64 restatement of the learned preconditioner's U-Net (test infrastructure).

Only the tests use this module, to check the library's network kernels
(``fs_unet_forward`` / ``fs_unet_gradient``) against it; it is never part of
the product path.  The network has no counterpart in the reference project (the
reference has no learned preconditioner), so this file restates the
library's own architecture in PyTorch CPU float64 with autograd:

* input channels: residual / RMS(residual over all nodes, free nodes summed),
  the three equilibrated edge masses, a fixed-node flag, 11 zero channels;
* encoder: per level two 3x3x3 convolutions (zero padding) with ReLU, then
  2x2x2 average pooling (ceil, mean over the children that exist);
* decoder: nearest upsampling, concatenation [upsampled | skip], two 3x3x3
  convolutions with ReLU;
* head: 1x1 convolution 16 -> 1; output 0 on fixed nodes;
* parameters in one vector theta laid out as the library's fs_unet_layer;
* loss: mean over samples of sum_free (out - t/scale)^2 / sum_free (t/scale)^2.

Convolution weights are rounded to BF16 before use, as the tensor-core
kernels consume them; everything else is FP64.
"""

from __future__ import annotations

import numpy as np

CIN = (16, 16, 16, 32, 32, 48, 48, 64, 112, 48, 80, 32, 48, 16)
COUT = (16, 16, 32, 32, 48, 48, 64, 64, 48, 48, 32, 32, 16, 16)


def layer_offsets():
    """(woff, boff) per convolution and the head offset, as fs_unet_layer."""
    offs = []
    o = 0
    for ci, co in zip(CIN, COUT):
        offs.append((o, o + 27 * ci * co))
        o += 27 * ci * co + co
    return offs, o


def param_count() -> int:
    return layer_offsets()[1] + 17


def init_theta(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, zero biases, small head (FP32)."""
    rng = np.random.default_rng(seed)
    offs, head = layer_offsets()
    th = np.zeros(param_count(), np.float32)
    for (wo, bo), ci, co in zip(offs, CIN, COUT):
        th[wo:bo] = rng.standard_normal(27 * ci * co) * np.sqrt(2.0 / (27 * ci))
    th[head:head + 16] = rng.standard_normal(16) * np.sqrt(1.0 / 16)
    return th


def _bf16(a):
    import torch
    return a.to(torch.bfloat16).to(a.dtype)


def forward(theta, rhs, em, label, dims, normalised=True):
    """theta (torch float64, requires_grad allowed), rhs (B, N), em (B, 3, N),
    label (B, N) uint8; returns (out (B, N), inv_scale (B,))."""
    import torch
    import torch.nn.functional as F
    B = rhs.shape[0]
    X, Y, Z = dims
    N = X * Y * Z
    free = torch.as_tensor(label == 0)
    rhs = torch.as_tensor(rhs, dtype=torch.float64)
    ss = (torch.where(free, rhs, torch.zeros_like(rhs)) ** 2).sum(dim=1)
    scale = torch.sqrt(ss / N)
    inv = torch.where(scale > 0, 1.0 / scale, torch.zeros_like(scale))
    x = torch.zeros((B, 16, X, Y, Z), dtype=torch.float64)
    x[:, 0] = torch.where(free, rhs * inv[:, None], torch.zeros_like(rhs)).reshape(B, X, Y, Z)
    emt = torch.as_tensor(em, dtype=torch.float64)
    x[:, 1:4] = emt.reshape(B, 3, X, Y, Z)
    x[:, 4] = (~free).to(torch.float64).reshape(B, X, Y, Z)
    offs, head = layer_offsets()

    def conv(l, v):
        wo, bo = offs[l]
        ci, co = CIN[l], COUT[l]
        w = _bf16(theta[wo:bo]).reshape(3, 3, 3, co, ci).permute(3, 4, 0, 1, 2)
        return torch.relu(F.conv3d(v, w, bias=theta[bo:bo + co], padding=1))

    def pool(v):
        # 2x2x2 mean over the children that exist (odd sizes: ceil)
        X_, Y_, Z_ = v.shape[2:]
        pad = (0, Z_ % 2, 0, Y_ % 2, 0, X_ % 2)
        s = F.avg_pool3d(F.pad(v, pad), 2, stride=2) * 8.0
        ones = F.pad(torch.ones((1, 1, X_, Y_, Z_), dtype=v.dtype), pad)
        return s / (F.avg_pool3d(ones, 2, stride=2) * 8.0)

    def up(v, shape):
        u = v.repeat_interleave(2, dim=2).repeat_interleave(2, dim=3).repeat_interleave(2, dim=4)
        return u[:, :, :shape[0], :shape[1], :shape[2]]

    e0 = conv(1, conv(0, x))
    e1 = conv(3, conv(2, pool(e0)))
    e2 = conv(5, conv(4, pool(e1)))
    e3 = conv(7, conv(6, pool(e2)))
    d2 = conv(9, conv(8, torch.cat([up(e3, e2.shape[2:]), e2], dim=1)))
    d1 = conv(11, conv(10, torch.cat([up(d2, e1.shape[2:]), e1], dim=1)))
    d0 = conv(13, conv(12, torch.cat([up(d1, e0.shape[2:]), e0], dim=1)))
    out = (d0 * theta[head:head + 16].reshape(1, 16, 1, 1, 1)).sum(dim=1) + theta[head + 16]
    out = out.reshape(B, N)
    out = torch.where(free, out, torch.zeros_like(out))
    if not normalised:
        out = out * scale[:, None]
    return out, inv


def loss_and_grad(theta_np, rhs, em, label, target, dims):
    """Loss and dLoss/dtheta in FP64 (autograd)."""
    import torch
    theta = torch.tensor(np.asarray(theta_np, np.float64), requires_grad=True)
    out, inv = forward(theta, rhs, em, label, dims, normalised=True)
    free = torch.as_tensor(label == 0)
    t = torch.as_tensor(target, dtype=torch.float64) * inv[:, None]
    z = torch.zeros_like(t)
    num = (torch.where(free, out - t, z) ** 2).sum(dim=1)
    den = (torch.where(free, t, z) ** 2).sum(dim=1)
    loss = (num / den).mean()
    loss.backward()
    return float(loss.detach()), theta.grad.numpy()
