"""TEST INFRASTRUCTURE: numpy restatement of the schedule network's forward
and backward passes (pscbfm_b200/csrc/bfm_mlp.cu), used only as the checker
of the CUDA kernels.

Network: in -> hidden -> hidden -> out, ReLU, parameters as one fp32 vector
[W1 (hidden x in), b1, W2 (hidden x hidden), b2, W3 (out x hidden), b3].
The device multiplies bf16 operands and accumulates in fp32; this oracle
rounds the same operands to bf16 (round to nearest even) at the same points
and accumulates in fp64.  Loss: sum over outputs of w_o (y - t)^2, averaged
over the batch.
"""
from __future__ import annotations

import numpy as np


ROUND = True  # False: exact fp64 arithmetic (for finite-difference checks of the formulas)


def bf16(x):
    """round to the nearest bf16 (ties to even), returned as float64"""
    if not ROUND:
        return np.asarray(x, np.float64)
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split(p, I, H, O):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((H, I), (H,), (H, H), (H,), (O, H), (O,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == p.size
    return out


def forward(p, x, I, H, O):
    W1, b1, W2, b2, W3, b3 = split(p, I, H, O)
    xb = bf16(x)
    h1 = np.maximum(xb @ bf16(W1).T + bf16_f32(b1), 0.0)
    h2 = np.maximum(bf16(h1) @ bf16(W2).T + bf16_f32(b2), 0.0)
    y = bf16(h2) @ bf16(W3).T + bf16_f32(b3)
    return y, (xb, h1, h2)


def bf16_f32(v):
    """biases stay fp32 on the device"""
    if not ROUND:
        return np.asarray(v, np.float64)
    return np.asarray(v, np.float32).astype(np.float64)


def gradients(p, x, t, w, I, H, O):
    """(loss, gradient vector) as the device computes them"""
    W1, b1, W2, b2, W3, b3 = split(p, I, H, O)
    M = x.shape[0]
    w = np.ones(O) if w is None else np.asarray(w, np.float64)
    y, (xb, h1, h2) = forward(p, x, I, H, O)
    d = y - np.asarray(t, np.float64)
    loss = float(np.sum(w * d * d) / M)
    dy = 2.0 * w * d / M
    dyb = bf16(dy)
    gW3 = dyb.T @ bf16(h2)
    gb3 = dy.sum(0)
    dh2 = (dyb @ bf16(W3)) * (h2 > 0)
    dh2b = bf16(dh2)
    gW2 = dh2b.T @ bf16(h1)
    gb2 = dh2.sum(0)
    dh1 = (dh2b @ bf16(W2)) * (h1 > 0)
    dh1b = bf16(dh1)
    gW1 = dh1b.T @ xb
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def adam(p, g, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """one Adam step (Kingma & Ba 2015); returns new (p, m1, m2)"""
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return p - lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps), m1, m2
