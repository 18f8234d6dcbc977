"""The U-Net of the learned stage, for training (inference runs in libvoxfea,
vf_learned.cu, with the same layer order and parameter layout).

  in (16 ch) -> [c0 16->16, c1 16->16] -> pool -> [c2 16->32, c3 32->32] -> pool
     -> [c4 32->64, c5 64->64] -> up -> c6 64->32 (+ skip) -> c7 32->32 -> up
     -> c8 32->16 (+ skip) -> c9 16->16 (FP32; channels 0..2 are the correction)

ReLU after every convolution but the last; skips are added before the ReLU.
Tensors are channels-last (Z, Y, X, C) BF16; every dimension of the input is a
multiple of 4.
"""

import numpy as np
import torch

from . import conv

LAYERS = ((16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 32), (32, 32), (32, 16), (16, 16))


def pool2(x):
    Z, Y, X, C = x.shape
    return x.float().view(Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(dim=(1, 3, 5)).to(torch.bfloat16)


def up2(x):
    return x.repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2).contiguous()


class UNet(torch.nn.Module):
    def __init__(self, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.w = torch.nn.ParameterList()
        self.b = torch.nn.ParameterList()
        for k, (ci, co) in enumerate(LAYERS):
            std = (2.0 / (27 * ci)) ** 0.5 * (0.1 if k == len(LAYERS) - 1 else 1.0)
            self.w.append(torch.nn.Parameter(torch.randn(27, co, ci, generator=g) * std))
            self.b.append(torch.nn.Parameter(torch.zeros(co)))

    def forward(self, x):
        c = conv.conv3d
        w, b = self.w, self.b
        relu = torch.relu
        a0 = relu(c(x, w[0], b[0]))
        s0 = relu(c(a0, w[1], b[1]))
        a1 = relu(c(pool2(s0), w[2], b[2]))
        s1 = relu(c(a1, w[3], b[3]))
        a2 = relu(c(pool2(s1), w[4], b[4]))
        b2 = relu(c(a2, w[5], b[5]))
        c1 = relu(c(up2(b2), w[6], b[6]) + s1)
        d1 = relu(c(c1, w[7], b[7]))
        c0 = relu(c(up2(d1), w[8], b[8]) + s0)
        return c(c0, w[9], b[9], out_f32=True)

    def flat_params(self):
        """FP32 vector in the libvoxfea layout: per layer W[27][cout][cin], b[cout]."""
        parts = []
        for w, b in zip(self.w, self.b):
            parts += [w.detach().float().cpu().reshape(-1), b.detach().float().cpu()]
        return torch.cat(parts).numpy().astype(np.float32)

    def load_flat(self, v):
        v = torch.as_tensor(np.asarray(v, dtype=np.float32))
        off = 0
        with torch.no_grad():
            for w, b in zip(self.w, self.b):
                nw = w.numel()
                w.copy_(v[off:off + nw].view_as(w))
                off += nw
                b.copy_(v[off:off + b.numel()])
                off += b.numel()
        assert off == v.numel()
