"""CPU FP32 reference of the learned preconditioner's network (torch
autograd), used to check the CUDA forward, backward and Adam kernels.

Activations are rounded to BF16 where the device stores them (after every
convolution, pooling and the input features), with a straight-through
gradient, so forward values are comparable element by element; the backward
is plain FP32 autograd.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F

LAYERS = [("e0a", 8, 32), ("e0b", 32, 32), ("e1a", 32, 64), ("e1b", 64, 64), ("ba", 64, 128),
          ("bb", 128, 128), ("d1a", 192, 64), ("d1b", 64, 64), ("d0a", 96, 32), ("d0b", 32, 32)]


def bf(t: torch.Tensor) -> torch.Tensor:
    """Round to BF16 and back, gradient passed straight through."""
    return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()


def conv_relu(x, w, b):
    """x [n,h,w,c], w [k,3,3,c] (KRSC), b [k] -> ReLU(conv + b) [n,h,w,k]."""
    y = F.conv2d(x.permute(0, 3, 1, 2), w.permute(0, 3, 1, 2), padding=1) + b[None, :, None, None]
    return torch.relu(y).permute(0, 2, 3, 1)


def pool(x):
    """2x2 average over the children that exist (ceil output sizes)."""
    n, h, w, c = x.shape
    ph, pw = h % 2, w % 2
    xp = F.pad(x, (0, 0, 0, pw, 0, ph))
    ones = F.pad(torch.ones(1, h, w, 1), (0, 0, 0, pw, 0, ph))
    s = xp.reshape(n, (h + ph) // 2, 2, (w + pw) // 2, 2, c).sum(dim=(2, 4))
    cnt = ones.reshape(1, (h + ph) // 2, 2, (w + pw) // 2, 2, 1).sum(dim=(2, 4))
    return s / cnt


def upcat(lo, skip):
    h, w = skip.shape[1], skip.shape[2]
    up = lo.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)[:, :h, :w]
    return torch.cat([up, skip], dim=-1)


def forward(params: dict, x: torch.Tensor) -> torch.Tensor:
    """params: name -> FP32 tensor (conv weights/biases BF16-valued);
    x [n,h,w,8] -> z [n*h*w]."""
    P = params

    def c(name, t):
        return bf(conv_relu(t, P[name + ".w"], P[name + ".b"]))

    e0 = c("e0b", c("e0a", x))
    e1 = c("e1b", c("e1a", bf(pool(e0))))
    b = c("bb", c("ba", bf(pool(e1))))
    d1 = c("d1b", c("d1a", upcat(b, e1)))
    d0 = c("d0b", c("d0a", upcat(d1, e0)))
    z = d0 @ P["head.w"] + P["head.b"]
    return z.reshape(-1)


def features(r, scale, feat_static):
    """[h*w] residual, [h*w*3] static channels -> [h*w, 8] BF16-valued."""
    npix = r.numel()
    x = torch.zeros(npix, 8)
    x[:, 0] = (r / scale).float()
    x[:, 1:4] = feat_static.reshape(npix, 3)
    return x.to(torch.bfloat16).to(torch.float32)
