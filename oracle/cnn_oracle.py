"""CPU oracle of the learned field correction's CNN -- TEST INFRASTRUCTURE.

A numpy restatement of the network the product runs on the tensor cores (octopus.jl_b200/csrc/cnn_host.cuh):
a 4-level U-Net of 3x3 / padding-1 convolutions with 32 base channels, ReLU, 2x2 average pooling, nearest
upsampling with skip concatenation, an 8-channel head whose channels 0 and 1 are the output, and the masked
mean-square loss.  The network has no counterpart in the reference (it corrects the reference's
Gaussian-subtracted hybrid, src/tasks/strongstrong/gaussian_pic.jl), so this file is its own specification.

`rounding=True` mirrors where the product rounds to bf16: the weights, every stored activation (after bias and
ReLU), the pooled maps, the loss gradient and every gradient a convolution reads; sums are float64 here
(float32 on the device).  `rounding=False` is plain float64 arithmetic, which the finite-difference test uses
to pin the backward pass itself.  Only tests import this module.
"""
from __future__ import annotations

import numpy as np

# (cin, cout, level, relu) per layer: e1a, e1b, e2a, e2b, e3a, e3b, b, d3, d2, d1, head
LAYERS = [(8, 32, 0, 1), (32, 32, 0, 1), (32, 64, 1, 1), (64, 64, 1, 1), (64, 128, 2, 1), (128, 128, 2, 1),
          (128, 128, 3, 1), (256, 64, 2, 1), (128, 32, 1, 1), (64, 32, 0, 1), (32, 8, 0, 0)]


def bf16(x):
    """Round to bfloat16 (round to nearest even) and return float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split_params(p):
    """The flat parameter vector as [(W [cout, 3, 3, cin], b [cout]), ...]."""
    out, off = [], 0
    for cin, cout, _, _ in LAYERS:
        n = cout * 9 * cin
        w = np.asarray(p[off:off + n], dtype=np.float64).reshape(cout, 3, 3, cin)
        off += n
        b = np.asarray(p[off:off + cout], dtype=np.float64)
        off += cout
        out.append((w, b))
    assert off == len(p)
    return out


def im2col(x):
    """x [B, H, W, C] -> [B*H*W, 9*C] with column (ky*3 + kx)*C + c, zero padding 1."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    cols = [xp[:, ky:ky + H, kx:kx + W, :] for ky in range(3) for kx in range(3)]
    return np.concatenate(cols, axis=3).reshape(B * H * W, 9 * C)


def col2im(d, shape):
    """Adjoint of im2col: d [B*H*W, 9*C] -> [B, H, W, C]."""
    B, H, W, C = shape
    d = d.reshape(B, H, W, 9, C)
    xp = np.zeros((B, H + 2, W + 2, C))
    for t in range(9):
        ky, kx = divmod(t, 3)
        xp[:, ky:ky + H, kx:kx + W, :] += d[:, :, :, t, :]
    return xp[:, 1:-1, 1:-1]


def pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 0::2] + x[:, 1::2, 1::2])


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_adj(d):
    return d[:, 0::2, 0::2] + d[:, 0::2, 1::2] + d[:, 1::2, 0::2] + d[:, 1::2, 1::2]


def pool_adj(d):
    return 0.25 * up(d)


class Net:
    def __init__(self, params, rounding=True):
        self.layers = split_params(params)
        self.r = bf16 if rounding else (lambda v: np.asarray(v, dtype=np.float64))

    def conv(self, k, x):
        w, b = self.layers[k]
        cout = w.shape[0]
        wq = self.r(w).reshape(cout, -1)
        return im2col(x) @ wq.T + b, wq

    def forward(self, x):
        """x [B, H, W, 8] (already bf16 values) -> head output [B, H, W, 8]; keeps what backward needs."""
        r = self.r
        B, H, W, _ = x.shape
        st = {"x0": x}

        def layer(k, inp):
            z, _ = self.conv(k, inp)
            relu = LAYERS[k][3]
            Hk, Wk = inp.shape[1], inp.shape[2]
            z = z.reshape(B, Hk, Wk, -1)
            return r(np.maximum(z, 0.0)) if relu else z

        st["a0"] = layer(0, x)
        st["s1"] = layer(1, st["a0"])
        st["p1"] = r(pool(st["s1"]))
        st["a2"] = layer(2, st["p1"])
        st["s2"] = layer(3, st["a2"])
        st["p2"] = r(pool(st["s2"]))
        st["a4"] = layer(4, st["p2"])
        st["s3"] = layer(5, st["a4"])
        st["p3"] = r(pool(st["s3"]))
        st["b6"] = layer(6, st["p3"])
        st["u3"] = np.concatenate([up(st["b6"]), st["s3"]], axis=3)
        st["d7"] = layer(7, st["u3"])
        st["u2"] = np.concatenate([up(st["d7"]), st["s2"]], axis=3)
        st["d8"] = layer(8, st["u2"])
        st["u1"] = np.concatenate([up(st["d8"]), st["s1"]], axis=3)
        st["d9"] = layer(9, st["u1"])
        st["out"] = layer(10, st["d9"])
        self.st = st
        return st["out"]

    def loss_and_grads(self, x, target, mask=None):
        """Masked mean-square loss of output channels 0..1 and the gradient of every parameter, flat."""
        r = self.r
        out = self.forward(x)
        st = self.st
        B, H, W, _ = x.shape
        w = np.ones((B, H, W)) if mask is None else np.asarray(mask, dtype=np.float64)
        wt = w.sum()
        d = out[..., :2] - target
        loss = float((w[..., None] * d * d).sum() / (2.0 * wt))
        g_out = np.zeros_like(out)
        g_out[..., :2] = 2.0 * w[..., None] * d / (2.0 * wt)
        g_out = r(g_out)
        grads = [None] * len(LAYERS)

        def back(k, inp, g, need_dx=True):
            """g: bf16 gradient of layer k's output; returns the input gradient (float)."""
            cout = LAYERS[k][1]
            gm = g.reshape(-1, cout)
            cols = im2col(inp)
            dw = (gm.T @ cols).reshape(self.layers[k][0].shape)
            db = gm.sum(axis=0)
            grads[k] = (dw, db)
            if not need_dx:
                return None
            wq = r(self.layers[k][0]).reshape(cout, -1)
            return col2im(gm @ wq, inp.shape)

        def relu_g(dy, y):
            return r(np.where(y > 0, dy, 0.0))

        dx = back(10, st["d9"], g_out)
        g = relu_g(dx, st["d9"])
        du1 = back(9, st["u1"], g)
        g = relu_g(up_adj(du1[..., :32]), st["d8"])
        ds1 = du1[..., 32:]
        du2 = back(8, st["u2"], g)
        g = relu_g(up_adj(du2[..., :64]), st["d7"])
        ds2 = du2[..., 64:]
        du3 = back(7, st["u3"], g)
        g = relu_g(up_adj(du3[..., :128]), st["b6"])
        ds3 = du3[..., 128:]
        dp3 = back(6, st["p3"], g)
        ds3 = ds3 + pool_adj(dp3)
        g = relu_g(ds3, st["s3"])
        da4 = back(5, st["a4"], g)
        g = relu_g(da4, st["a4"])
        dp2 = back(4, st["p2"], g)
        ds2 = ds2 + pool_adj(dp2)
        g = relu_g(ds2, st["s2"])
        da2 = back(3, st["a2"], g)
        g = relu_g(da2, st["a2"])
        dp1 = back(2, st["p1"], g)
        ds1 = ds1 + pool_adj(dp1)
        g = relu_g(ds1, st["s1"])
        da0 = back(1, st["a0"], g)
        g = relu_g(da0, st["a0"])
        back(0, st["x0"], g, need_dx=False)
        flat = np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])
        return loss, flat


def num_params():
    return sum(cout * 9 * cin + cout for cin, cout, _, _ in LAYERS)
