"""CPU restatement of the learned-guess U-Net (test infrastructure only).

Not part of the product: the tests use it to check the device network
(``cism_b200/net.py`` over ``libbpnet.so``) -- its forward pass and every
weight and bias gradient -- on the same weights and inputs.  The device
rounds to BF16 at fixed points (the input, the GEMM copies of the weights,
every activation after its nonlinearity, and the pre-activation gradient
fed to the two gradient GEMMs); ``bf16=True`` rounds at the same points and
computes everything else in FP64, so the two differ by FP32 accumulation
only.  With ``bf16=False`` the restatement is plain FP64, for the
finite-difference check of its own gradients.

Layout and conventions follow the device: NHWC, weights [Cout][9 Cin] with
k = tap * Cin + c and tap = (dy + 1) * 3 + (dx + 1), periodic or zero
borders, GELU(x) = x Phi(x), 2 x 2 average pooling, nearest upsampling,
decoder input = [upsampled | skip] along channels, a 1 x 1 linear head.
"""
from __future__ import annotations

import math

import numpy as np

try:  # erf for arrays
    from scipy.special import erf as _erf
except Exception:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to BF16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _erf(x / math.sqrt(2.0)))
    return cdf + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def _shift(x, dy, dx, periodic):
    """out[y][x] = in[y + dy][x + dx] (periodic or zero outside)."""
    if periodic:
        return np.roll(np.roll(x, -dy, axis=1), -dx, axis=2)
    B, H, W, C = x.shape
    out = np.zeros_like(x)
    ys = slice(max(0, -dy), min(H, H - dy))
    xs = slice(max(0, -dx), min(W, W - dx))
    yd = slice(max(0, dy), min(H, H + dy))
    xd = slice(max(0, dx), min(W, W + dx))
    out[:, ys, xs] = x[:, yd, xd]
    return out


def im2col(x, periodic):
    taps = [_shift(x, t // 3 - 1, t % 3 - 1, periodic) for t in range(9)]
    return np.concatenate(taps, axis=-1)  # [B][H][W][9 C], k = tap * C + c


def col2im(dcol, C, periodic):
    dx = 0.0
    for t in range(9):
        dx = dx + _shift(dcol[..., t * C:(t + 1) * C], -(t // 3 - 1), -(t % 3 - 1), periodic)
    return dx


def pool(x):
    return 0.25 * (x[:, 0::2, 0::2] + x[:, 1::2, 0::2] + x[:, 0::2, 1::2] + x[:, 1::2, 1::2])


def pool_grad(dy):
    return 0.25 * np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2)


def up(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up_grad(dy):
    return dy[:, 0::2, 0::2] + dy[:, 1::2, 0::2] + dy[:, 0::2, 1::2] + dy[:, 1::2, 1::2]


class OracleUNet:
    """Same structure as the device network; weights are lists of
    (w [Cout][K], b [Cout], k3, act) in the device's order: encoder convs,
    decoder convs (deepest first), head."""

    def __init__(self, convs, channels, n_in=5, bf16_points=True):
        self.convs = convs
        self.channels = list(channels)
        self.n_in = n_in
        self.r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))

    def _conv(self, i, x, periodic, cache):
        w, b, k3, act = self.convs[i]
        col = im2col(x, periodic) if k3 else x
        z = col @ self.r(w).T + b
        y = self.r(gelu(z)) if act else z
        cache[i] = (col, z, x.shape)
        return y, z

    def forward(self, x, periodic):
        cache = {}
        cur = self.r(x)
        nl = len(self.channels)
        i = 0
        skips = []
        for lv in range(nl):
            if lv > 0:
                cur = self.r(pool(cur))
            for _ in range(2):
                cur, _ = self._conv(i, cur, periodic, cache)
                i += 1
            skips.append(cur)
        for lv in range(nl - 2, -1, -1):
            cur = np.concatenate([up(cur), skips[lv]], axis=-1)
            for _ in range(2):
                cur, _ = self._conv(i, cur, periodic, cache)
                i += 1
        _, z = self._conv(i, cur, periodic, cache)
        self.cache = cache
        return z

    def _conv_back(self, i, dy, periodic, grads, need_dx):
        w, b, k3, act = self.convs[i]
        col, z, xshape = self.cache[i]
        dz = dy * gelu_grad(z) if act else dy
        grads[i] = (None, dz.sum(axis=(0, 1, 2)))
        dzr = self.r(dz)
        K = col.shape[-1]
        gw = dzr.reshape(-1, dz.shape[-1]).T @ col.reshape(-1, K)
        grads[i] = (gw, grads[i][1])
        if not need_dx:
            return None
        dcol = dzr @ self.r(w)
        return col2im(dcol, xshape[-1], periodic) if k3 else dcol

    def backward(self, dout, periodic):
        grads = {}
        nl = len(self.channels)
        nconv = len(self.convs)
        i = nconv - 1
        d = self._conv_back(i, dout, periodic, grads, True)
        i -= 1
        dskip = [None] * nl
        for lv in range(nl - 1):
            d = self._conv_back(i, d, periodic, grads, True)
            d = self._conv_back(i - 1, d, periodic, grads, True)
            i -= 2
            cu = self.channels[lv + 1]
            dskip[lv] = d[..., cu:]
            d = up_grad(d[..., :cu])
        for lv in range(nl - 1, -1, -1):
            if lv < nl - 1:
                d = dskip[lv]
            d = self._conv_back(i, d, periodic, grads, True)
            d = self._conv_back(i - 1, d, periodic, grads, lv > 0)
            i -= 2
            if lv > 0:
                dskip[lv - 1] = dskip[lv - 1] + pool_grad(d)
        return [grads[k] for k in range(nconv)]
