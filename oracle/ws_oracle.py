"""CPU restatement of the warm-start network (caustic_b200/warmstart.py) for
the gradient checks.  Test infrastructure only: nothing in the product calls
it.

Same conventions as the GPU path: NHWC activations, weights [cout][9*cin]
with column tap*cin + c (tap = (dy+1)*3 + (dx+1), zero padding 1), 2x2 mean
pooling, nearest upsampling, decoder input = [upsampled, skip] channels, a
1x1 head to 8 outputs of which channel 0 is the prediction, and the
mean-free squared-error loss.  Values are rounded to bfloat16 where the GPU
path stores them in bfloat16 (activations, weights, and the gradients fed to
the GEMMs); sums are in float64.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def im2col(x):
    """x [B,H,W,C] -> [B*H*W, 9*C]"""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    cols = np.empty((B, H, W, 9, C))
    for tap in range(9):
        dy, dx = tap // 3, tap % 3
        cols[:, :, :, tap] = xp[:, dy:dy + H, dx:dx + W]
    return cols.reshape(B * H * W, 9 * C)


def col2im(dcols, shape):
    B, H, W, C = shape
    d = dcols.reshape(B, H, W, 9, C)
    dxp = np.zeros((B, H + 2, W + 2, C))
    for tap in range(9):
        dy, dx = tap // 3, tap % 3
        dxp[:, dy:dy + H, dx:dx + W] += d[:, :, :, tap]
    return dxp[:, 1:-1, 1:-1]


def pool2(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def pool2_back(d, shape):
    return np.repeat(np.repeat(d, 2, axis=1), 2, axis=2) * 0.25


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up2_back(d):
    B, H, W, C = d.shape
    return d.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


class Net:
    """params: list of (w [cout][fan], b or None) in the GPU layer order:
    encoder convs, decoder convs, head."""

    def __init__(self, params, levels, ch):
        self.params = params
        self.levels = levels
        self.ch = ch

    def _conv(self, k, x, relu=True, one=False):
        w, b = self.params[k]
        B, H, W, C = x.shape
        cols = x.reshape(B * H * W, C) if one else im2col(x)
        d = cols @ bf16(w).T
        if b is None:
            return d.reshape(B, H, W, -1), (cols, None, x.shape)
        pre = d + b
        y = np.maximum(pre, 0.0) if relu else pre
        return bf16(y).reshape(B, H, W, -1), (cols, pre, x.shape)

    def forward(self, x):
        tape = []
        k = 0
        h = bf16(x)
        skips = []
        for l in range(self.levels):
            for _ in range(2):
                h, t = self._conv(k, h)
                tape.append(t)
                k += 1
            skips.append(h)
            if l < self.levels - 1:
                h = bf16(pool2(h))
        for l in range(self.levels - 2, -1, -1):
            h = np.concatenate([up2(h), skips[l]], axis=3)
            for _ in range(2):
                h, t = self._conv(k, h)
                tape.append(t)
                k += 1
        d, t = self._conv(k, h, one=True)
        tape.append(t)
        self.tape = tape
        B, H, W, _ = d.shape
        return d[..., 0].reshape(B, H * W)

    def backward(self, dpred):
        grads = [None] * len(self.params)
        k = len(self.params) - 1
        cols, _, shape = self.tape[k]
        B, H, W, C = shape
        dd = np.zeros((B * H * W, 8))
        dd[:, 0] = dpred.reshape(-1)
        dz = bf16(dd)
        grads[k] = (dz.T @ cols, None)
        dh = (dz @ bf16(self.params[k][0])).reshape(B, H, W, C)
        k -= 1

        def conv_back(k, dh):
            cols, pre, shape = self.tape[k]
            g = dh.reshape(pre.shape) * (pre > 0)
            dz = bf16(g)
            grads[k] = (dz.T @ cols, g.sum(axis=0))
            return col2im(dz @ bf16(self.params[k][0]), shape)

        dskip = [None] * self.levels
        for l in range(self.levels - 1):
            for _ in range(2):
                dh = conv_back(k, dh)
                k -= 1
            c1 = self.ch[l + 1]
            dskip[l] = dh[..., c1:]
            dh = up2_back(dh[..., :c1])
        for l in range(self.levels - 1, -1, -1):
            if l < self.levels - 1:
                dh = pool2_back(dh, None) + dskip[l]
            for _ in range(2):
                dh = conv_back(k, dh)
                k -= 1
        assert k == -1
        return grads


def loss_grad(pred, target, grid=None, lam=0.0):
    """Mean-free squared error with lam weighing the squared differences
    between grid neighbours (grid = (gy, gx), row-major; default square)."""
    B, n = pred.shape
    gy, gx = grid if grid else (int(round(np.sqrt(n))),) * 2
    e = pred - target
    e = e - e.mean(axis=1, keepdims=True)
    E = e.reshape(B, gy, gx)
    dx = E[:, :, 1:] - E[:, :, :-1]
    dy = E[:, 1:, :] - E[:, :-1, :]
    loss = ((e * e).sum() + lam * ((dx * dx).sum() + (dy * dy).sum())) / (n * B)
    G = 2.0 * E
    G[:, :, 1:] += 2.0 * lam * dx
    G[:, :, :-1] -= 2.0 * lam * dx
    G[:, 1:, :] += 2.0 * lam * dy
    G[:, :-1, :] -= 2.0 * lam * dy
    return float(loss), G.reshape(B, n) / (n * B)
