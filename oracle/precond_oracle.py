"""CPU oracle of the learned preconditioner's network (test infrastructure).

Only tests, the smoke check and the benchmark's CPU legs use this module,
as the checker of the library's CUDA kernels; nothing in the product calls
it.  The network has no counterpart in the reference, so this is a plain
torch FP32 (CPU) restatement of the same computation:

* the 4-level encoder-decoder of ``swfwi_b200/csrc/precond.hpp`` on NHWC
  images, weights [cout][3][3][cin] in one flat FP32 vector;
* with ``bf16=True`` the values are rounded to BF16 exactly where the GPU
  stores BF16: the padded input, every conv weight, every conv output (after
  bias and ReLU), the pooled maps and the ReLU-masked output gradients that
  feed the tensor-core products; sums stay FP32;
* the backward pass is written out by hand in the GPU's order (output
  layer, then each decoder level, the bottleneck and the encoder, with the
  skip gradients from the concatenations and the pools added), so that with
  ``bf16=False`` it can be checked against torch autograd.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F


def bf(x: torch.Tensor) -> torch.Tensor:
    return x.to(torch.bfloat16).to(torch.float32)


def layer_table(widths=(16, 32, 64, 64)):
    """[(cin, cout, w_off, b_off)] of the 14 convs and the output layer, in
    the library's flat order."""
    c0, c1, c2, c3 = widths
    io = [(16, c0), (c0, c0), (c0, c1), (c1, c1), (c1, c2), (c2, c2), (c2, c3), (c3, c3),
          (c3 + c2, c2), (c2, c2), (c2 + c1, c1), (c1, c1), (c1 + c0, c0), (c0, c0)]
    out, off = [], 0
    for ci, co in io:
        w = off
        off += co * 9 * ci
        out.append((ci, co, w, off))
        off += co
    out.append((c0, 1, off, off + c0))
    return out, off + c0 + 1


class NetOracle:
    def __init__(self, params: np.ndarray, widths=(16, 32, 64, 64), bf16: bool = True):
        self.widths = tuple(widths)
        self.layers, n = layer_table(widths)
        assert params.size == n, (params.size, n)
        self.p = torch.from_numpy(np.asarray(params, np.float32).copy())
        self.bf16 = bf16

    def _r(self, x):
        return bf(x) if self.bf16 else x

    def weight(self, l):
        ci, co, wo, bo = self.layers[l]
        w = self.p[wo:wo + co * 9 * ci].reshape(co, 3, 3, ci).permute(0, 3, 1, 2).contiguous()
        return self._r(w), self.p[bo:bo + co]

    # NHWC <-> NCHW
    @staticmethod
    def _c(x):
        return x.permute(0, 3, 1, 2).contiguous()

    @staticmethod
    def _h(x):
        return x.permute(0, 2, 3, 1).contiguous()

    def conv(self, l, a):
        w, b = self.weight(l)
        z = self._h(F.conv2d(self._c(a), w, padding=1)) + b
        return self._r(torch.relu(z))

    def pool(self, a):
        s = ((a[:, 0::2, 0::2] + a[:, 0::2, 1::2]) + a[:, 1::2, 0::2]) + a[:, 1::2, 1::2]
        return self._r(s * 0.25)

    @staticmethod
    def upcat(low, skip):
        up = low.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)
        return torch.cat([up, skip], dim=3)

    def forward(self, x3: np.ndarray) -> np.ndarray:
        x = torch.from_numpy(np.asarray(x3, np.float32))
        N, H, W, _ = x.shape
        x16 = torch.zeros((N, H, W, 16))
        x16[..., :3] = x
        x16 = self._r(x16)
        A = {"x16": x16}
        A["a0"] = self.conv(0, x16)
        A["s0"] = self.conv(1, A["a0"])
        A["p0"] = self.pool(A["s0"])
        A["a1"] = self.conv(2, A["p0"])
        A["s1"] = self.conv(3, A["a1"])
        A["p1"] = self.pool(A["s1"])
        A["a2"] = self.conv(4, A["p1"])
        A["s2"] = self.conv(5, A["a2"])
        A["p2"] = self.pool(A["s2"])
        A["a3"] = self.conv(6, A["p2"])
        A["b3"] = self.conv(7, A["a3"])
        A["cat2"] = self.upcat(A["b3"], A["s2"])
        A["a4"] = self.conv(8, A["cat2"])
        A["u2"] = self.conv(9, A["a4"])
        A["cat1"] = self.upcat(A["u2"], A["s1"])
        A["a5"] = self.conv(10, A["cat1"])
        A["u1"] = self.conv(11, A["a5"])
        A["cat0"] = self.upcat(A["u1"], A["s0"])
        A["a6"] = self.conv(12, A["cat0"])
        A["u0"] = self.conv(13, A["a6"])
        ci, _, wo, bo = self.layers[14]
        A["y"] = (A["u0"] * self.p[wo:wo + ci]).sum(-1) + self.p[bo]
        self.A = A
        return A["y"].numpy()

    def _conv_bwd(self, l, a_in, a_out, dY, grads, need_dx=True):
        ci, co, wo, bo = self.layers[l]
        dz = dY * (a_out > 0).to(torch.float32)
        dz = self._r(dz)
        grads[bo:bo + co] += dz.sum(dim=(0, 1, 2))
        dw = torch.nn.grad.conv2d_weight(self._c(a_in), (co, ci, 3, 3), self._c(dz), padding=1)
        grads[wo:wo + co * 9 * ci] += dw.permute(0, 2, 3, 1).reshape(-1)
        if not need_dx:
            return None
        w, _ = self.weight(l)
        return self._h(torch.nn.grad.conv2d_input(tuple(self._c(a_in).shape), w, self._c(dz), padding=1))

    @staticmethod
    def _upcat_bwd(dcat, c1):
        d = dcat[..., :c1]
        low = ((d[:, 0::2, 0::2] + d[:, 0::2, 1::2]) + d[:, 1::2, 0::2]) + d[:, 1::2, 1::2]
        return low, dcat[..., c1:].clone()

    @staticmethod
    def _pool_bwd(dp):
        return 0.25 * dp.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)

    def backward(self, t: np.ndarray):
        """Mean-square loss of the last forward against t and the flat
        parameter gradient."""
        A = self.A
        c0, c1, c2, c3 = self.widths
        tt = torch.from_numpy(np.asarray(t, np.float32))
        r = A["y"] - tt
        P = r.numel()
        loss = float((r.double() ** 2).sum() / P)
        dy = (2.0 / P) * r
        grads = torch.zeros_like(self.p)
        ci, _, wo, bo = self.layers[14]
        grads[wo:wo + ci] = (A["u0"] * dy[..., None]).sum(dim=(0, 1, 2))
        grads[bo] = dy.sum()
        d = dy[..., None] * self.p[wo:wo + ci]
        d = self._conv_bwd(13, A["a6"], A["u0"], d, grads)
        d = self._conv_bwd(12, A["cat0"], A["a6"], d, grads)
        dlow, ds0 = self._upcat_bwd(d, c1)
        d = self._conv_bwd(11, A["a5"], A["u1"], dlow, grads)
        d = self._conv_bwd(10, A["cat1"], A["a5"], d, grads)
        dlow, ds1 = self._upcat_bwd(d, c2)
        d = self._conv_bwd(9, A["a4"], A["u2"], dlow, grads)
        d = self._conv_bwd(8, A["cat2"], A["a4"], d, grads)
        dlow, ds2 = self._upcat_bwd(d, c3)
        d = self._conv_bwd(7, A["a3"], A["b3"], dlow, grads)
        d = self._conv_bwd(6, A["p2"], A["a3"], d, grads)
        ds2 = ds2 + self._pool_bwd(d)
        d = self._conv_bwd(5, A["a2"], A["s2"], ds2, grads)
        d = self._conv_bwd(4, A["p1"], A["a2"], d, grads)
        ds1 = ds1 + self._pool_bwd(d)
        d = self._conv_bwd(3, A["a1"], A["s1"], ds1, grads)
        d = self._conv_bwd(2, A["p0"], A["a1"], d, grads)
        ds0 = ds0 + self._pool_bwd(d)
        d = self._conv_bwd(1, A["a0"], A["s0"], ds0, grads)
        self._conv_bwd(0, A["x16"], A["a0"], d, grads, need_dx=False)
        return loss, grads.numpy()


def autograd_reference(params: np.ndarray, x3: np.ndarray, t: np.ndarray, widths=(16, 32, 64, 64)):
    """Loss and parameter gradient by torch autograd of the FP32 network (no
    BF16 rounding): the check of NetOracle's hand-written backward."""
    layers, n = layer_table(widths)
    p = torch.from_numpy(np.asarray(params, np.float32).copy()).requires_grad_(True)
    x = torch.from_numpy(np.asarray(x3, np.float32))
    N, H, W, _ = x.shape
    x16 = torch.cat([x, torch.zeros((N, H, W, 13))], dim=3).permute(0, 3, 1, 2)

    def conv(l, a):
        ci, co, wo, bo = layers[l]
        w = p[wo:wo + co * 9 * ci].reshape(co, 3, 3, ci).permute(0, 3, 1, 2)
        return torch.relu(F.conv2d(a, w, p[bo:bo + co], padding=1))

    def pool(a):
        return F.avg_pool2d(a, 2)

    def up(a):
        return F.interpolate(a, scale_factor=2, mode="nearest")

    s0 = conv(1, conv(0, x16))
    s1 = conv(3, conv(2, pool(s0)))
    s2 = conv(5, conv(4, pool(s1)))
    b3 = conv(7, conv(6, pool(s2)))
    u2 = conv(9, conv(8, torch.cat([up(b3), s2], 1)))
    u1 = conv(11, conv(10, torch.cat([up(u2), s1], 1)))
    u0 = conv(13, conv(12, torch.cat([up(u1), s0], 1)))
    ci, _, wo, bo = layers[14]
    y = (u0 * p[wo:wo + ci].reshape(1, ci, 1, 1)).sum(1) + p[bo]
    tt = torch.from_numpy(np.asarray(t, np.float32))
    loss = ((y - tt) ** 2).mean()
    loss.backward()
    return float(loss), y.detach().numpy(), p.grad.numpy()
