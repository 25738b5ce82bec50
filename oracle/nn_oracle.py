"""CPU restatement of the warm-start network (numpy, float64).

TEST INFRASTRUCTURE: the checker for the tensor-core network kernels
(atlaswerks_b200/csrc/nn.cu) and for the gradients of the host network
(atlaswerks_b200/warmstart.py). The network has no counterpart in the
reference; this module states the same operations directly:

* 3x3x3 (or 1x1x1) zero-padded convolution, channels last:
  y[p][co] = sum_{tap,ci} x[p + off(tap)][ci] w[co][tap][ci] + b[co],
  off(tap) = (tap // 9 - 1, tap // 3 % 3 - 1, tap % 3 - 1) as (dz, dy, dx);
  its data gradient dx[p][ci] = sum dy[p - off(tap)][co] w[co][tap][ci] and
  weight gradient dw[co][tap][ci] = sum_p dy[p][co] x[p + off(tap)][ci];
* ReLU, 2x2x2 average pooling, nearest x2 upsampling, channel concatenation;
* the MSE of the first three output channels.

Values pass through bf16() where the device stores BF16, so a comparison
measures accumulation and rounding order only.
"""
from __future__ import annotations

import numpy as np


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def offsets(ntaps: int):
    if ntaps == 1:
        return [(0, 0, 0)]
    return [(t // 9 - 1, t // 3 % 3 - 1, t % 3 - 1) for t in range(27)]


def shift(x: np.ndarray, off, sign: int = 1) -> np.ndarray:
    """s[b, z, y, x] = x[b, z + sign*dz, y + sign*dy, x + sign*dx], zero outside."""
    dz, dy, dx = (sign * o for o in off)
    B, D, H, W, C = x.shape
    out = np.zeros_like(x)
    zs, ys, xs = slice(max(0, -dz), min(D, D - dz)), slice(max(0, -dy), min(H, H - dy)), \
        slice(max(0, -dx), min(W, W - dx))
    zt, yt, xt = slice(max(0, dz), min(D, D + dz)), slice(max(0, dy), min(H, H + dy)), \
        slice(max(0, dx), min(W, W + dx))
    out[:, zs, ys, xs] = x[:, zt, yt, xt]
    return out


def conv_fwd(x, w, b=None, relu=False):
    """x [B,D,H,W,Cin], w [Cout,taps,Cin] -> [B,D,H,W,Cout] (float64)."""
    x = x.astype(np.float64)
    w = w.astype(np.float64)
    y = np.zeros(x.shape[:4] + (w.shape[0],))
    for t, off in enumerate(offsets(w.shape[1])):
        y += shift(x, off) @ w[:, t, :].T
    if b is not None:
        y += b
    return np.maximum(y, 0.0) if relu else y


def conv_dgrad(dy, w, mask=None):
    dy = dy.astype(np.float64)
    w = w.astype(np.float64)
    dx = np.zeros(dy.shape[:4] + (w.shape[2],))
    for t, off in enumerate(offsets(w.shape[1])):
        dx += shift(dy, off, -1) @ w[:, t, :]
    if mask is not None:
        dx = dx * (mask > 0)
    return dx


def conv_wgrad(x, dy, ntaps):
    x = x.astype(np.float64)
    dy = dy.astype(np.float64)
    co, ci = dy.shape[-1], x.shape[-1]
    dw = np.zeros((co, ntaps, ci))
    d2 = dy.reshape(-1, co)
    for t, off in enumerate(offsets(ntaps)):
        dw[:, t, :] = d2.T @ shift(x, off).reshape(-1, ci)
    return dw


def pool(x):
    B, D, H, W, C = x.shape
    return x.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def pool_bwd(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_bwd(dy):
    B, D, H, W, C = dy.shape
    return dy.reshape(B, D // 2, 2, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4, 6))


class UNetOracle:
    """The encoder-decoder of atlaswerks_b200.warmstart (same layer list),
    forward and backward in float64 from given float32 weights."""

    def __init__(self, layers, weights, biases, store_bf16=True):
        self.layers = layers          # [(name, cin, cout, taps, relu)]
        # round the stored activations to BF16 as the device does (off for
        # finite-difference checks, which need a smooth forward)
        self.store_bf16 = store_bf16
        self.w = {n: bf16(weights[n]).astype(np.float64) for n, *_ in layers}
        self.b = {n: biases[n].astype(np.float64) for n, *_ in layers}

    def forward(self, x):
        a = {}
        # activations are stored in BF16 on the device; the head output in FP32
        rnd = ((lambda t: bf16(t.astype(np.float32)).astype(np.float64)) if self.store_bf16
               else (lambda t: t))
        c = lambda n, inp: (conv_fwd(inp, self.w[n], self.b[n], relu=False) if n == "head"
                            else rnd(conv_fwd(inp, self.w[n], self.b[n], relu=True)))
        pool_ = lambda t: rnd(pool(t))
        a["in"] = x
        a["e0a"] = c("e0a", x)
        a["e0b"] = c("e0b", a["e0a"])
        a["p0"] = pool_(a["e0b"])
        a["e1a"] = c("e1a", a["p0"])
        a["e1b"] = c("e1b", a["e1a"])
        a["p1"] = pool_(a["e1b"])
        a["e2a"] = c("e2a", a["p1"])
        a["e2b"] = c("e2b", a["e2a"])
        a["p2"] = pool_(a["e2b"])
        a["e3a"] = c("e3a", a["p2"])
        a["e3b"] = c("e3b", a["e3a"])
        a["c2"] = np.concatenate([up(a["e3b"]), a["e2b"]], -1)
        a["d2a"] = c("d2a", a["c2"])
        a["d2b"] = c("d2b", a["d2a"])
        a["c1"] = np.concatenate([up(a["d2b"]), a["e1b"]], -1)
        a["d1a"] = c("d1a", a["c1"])
        a["d1b"] = c("d1b", a["d1a"])
        a["c0"] = np.concatenate([up(a["d1b"]), a["e0b"]], -1)
        a["d0a"] = c("d0a", a["c0"])
        a["d0b"] = c("d0b", a["d0a"])
        a["out"] = c("head", a["d0b"])
        self.a = a
        return a["out"]

    def backward(self, dout):
        """dout: gradient of the head output [..., 16]. Returns {name: (dw, db)}."""
        a, g = self.a, {}

        def layer(n, inp, dy_pre, mask):
            g[n] = (conv_wgrad(inp, dy_pre, self.w[n].shape[1]), dy_pre.reshape(-1, dy_pre.shape[-1]).sum(0))
            return conv_dgrad(dy_pre, self.w[n], mask)

        relu_d = lambda d, y: d * (y > 0)
        d = layer("head", a["d0b"], dout, a["d0b"])
        d = layer("d0b", a["d0a"], d, a["d0a"])
        dc0 = layer("d0a", a["c0"], d, a["c0"])
        c_up = a["d1b"].shape[-1]
        d = up_bwd(dc0[..., :c_up])
        d = layer("d1b", a["d1a"], d, a["d1a"])
        dc1 = layer("d1a", a["c1"], d, a["c1"])
        c_up = a["d2b"].shape[-1]
        d = up_bwd(dc1[..., :c_up])
        d = layer("d2b", a["d2a"], d, a["d2a"])
        dc2 = layer("d2a", a["c2"], d, a["c2"])
        c_up = a["e3b"].shape[-1]
        d = up_bwd(dc2[..., :c_up])
        d = layer("e3b", a["e3a"], d, a["e3a"])
        dp2 = layer("e3a", a["p2"], d, None)
        d = relu_d(pool_bwd(dp2) + dc2[..., c_up:], a["e2b"])
        d = layer("e2b", a["e2a"], d, a["e2a"])
        dp1 = layer("e2a", a["p1"], d, None)
        c_skip1 = a["e1b"].shape[-1]
        d = relu_d(pool_bwd(dp1) + dc1[..., -c_skip1:], a["e1b"])
        d = layer("e1b", a["e1a"], d, a["e1a"])
        dp0 = layer("e1a", a["p0"], d, None)
        c_skip0 = a["e0b"].shape[-1]
        d = relu_d(pool_bwd(dp0) + dc0[..., -c_skip0:], a["e0b"])
        d = layer("e0b", a["e0a"], d, a["e0a"])
        layer("e0a", a["in"], d, None)
        return g
