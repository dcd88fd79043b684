"""TEST INFRASTRUCTURE ONLY -- float64 restatement of the schedule picker's
network (anionpy_b200/csrc/ionp_mlp.cu): forward pass and the gradients of
the mean squared error, in the library's flat parameter layout
W1[nin][h], b1[h], W2[h][h], b2[h], W3[h][nout], b3[nout]. The GPU kernels'
gradients are checked against it; it is itself checked against finite
differences (tests/test_cpu_picker_ref.py)."""
from __future__ import annotations

import numpy as np


def unpack(p, nin, h, nout):
    p = np.asarray(p, np.float64)
    sizes = [nin * h, h, h * h, h, h * nout, nout]
    out, o = [], 0
    for sz in sizes:
        out.append(p[o: o + sz])
        o += sz
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(nin, h), b1, W2.reshape(h, h), b2, W3.reshape(h, nout), b3


def forward(p, x, nin, h, nout):
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, h, nout)
    x = np.asarray(x, np.float64)
    h1 = np.maximum(x @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ W3 + b3, (h1, h2)


def loss_and_grads(p, x, t, nin, h, nout, mask=None):
    """(mean squared error, flat gradient) in float64."""
    W1, b1, W2, b2, W3, b3 = unpack(p, nin, h, nout)
    x = np.asarray(x, np.float64)
    y, (h1, h2) = forward(p, x, nin, h, nout)
    m = np.ones_like(y) if mask is None else np.asarray(mask, np.float64)
    d = (y - np.asarray(t, np.float64)) * m
    cnt = y.size
    loss = float((d * d).sum() / cnt)
    dy = 2.0 * d / cnt
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    dh2 = (dy @ W3.T) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = x.T @ dh1
    gb1 = dh1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
