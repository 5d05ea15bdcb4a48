"""TEST INFRASTRUCTURE ONLY -- FP64 numpy restatement of the selector
network (16-64-64-12, ReLU) used to check the GPU forward/backward kernels.

The GPU kernels take the weights and inputs in BF16 and accumulate in FP32;
this oracle applies the same BF16 rounding to weights and inputs and then
computes everything in FP64.  The network has no counterpart in the
reference.
"""
import numpy as np


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    x = ((x + 0x7FFF + ((x >> 16) & 1)) >> 16) << 16
    return x.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    o, out = 0, []
    for shape in ((64, 16), (64,), (64, 64), (64,), (12, 64), (12,)):
        k = int(np.prod(shape))
        out.append(np.asarray(p[o:o + k], dtype=np.float64).reshape(shape))
        o += k
    return out


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    W1, W2, W3 = bf16(W1), bf16(W2), bf16(W3)
    b1, b2, b3 = (np.asarray(b, dtype=np.float32).astype(np.float64) for b in (b1, b2, b3))
    x = bf16(x)
    h1 = np.maximum(x @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return x, h1, h2, h2 @ W3.T + b3


def loss_and_grad(p, x, t, mask=None):
    """Loss = mean over rows of sum_o mask (y - t)^2, and d loss / d p."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    W2q, W3q = bf16(W2), bf16(W3)
    xq, h1, h2, y = forward(p, x)
    m = np.ones_like(y) if mask is None else np.asarray(mask, dtype=np.float64)
    n = x.shape[0]
    e = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(m * e * e) / n)
    dy = 2 * m * e / n
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ W3q) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2q) * (h1 > 0)
    gW1 = d1.T @ xq
    gb1 = d1.sum(0)
    return loss, np.concatenate([g.ravel() for g in (gW1, gb1, gW2, gb2, gW3, gb3)])
