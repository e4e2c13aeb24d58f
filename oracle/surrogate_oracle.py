"""CPU oracle of the learned warm start's network (test infrastructure only).

Float64 NumPy restatement of the forward and backward pass that
water_flow_simulation_b200/surrogate.py runs on the tensor cores, used to check the GPU
loss and gradients.  The network has no counterpart in the reference (floodsim starts
every run from its 1D inlet profile, floodsim/lbm3d.py:362-364).

Layout: activations (V, C) channels-last on a (Z, Y, X) grid, voxel v = x + X*(y + Y*z);
conv weights (Cout, 27*Cin) with tap t = (dz+1)*9 + (dy+1)*3 + (dx+1) and zero padding.
Graph:  a1 = relu(c1 x);  p = pool2(a1);  a4 = relu(c4 relu(c3 relu(c2 p)));
        u = up2(a4) + a1;  out = c6 relu(c5 u);  loss = sum mask * (out[:, :4] - t)^2 / n.
"""
from __future__ import annotations

import numpy as np

LAYERS = (("c1", 8, 64, True), ("c2", 64, 128, True), ("c3", 128, 128, True), ("c4", 128, 64, True),
          ("c5", 64, 64, True), ("c6", 64, 8, False))


def _taps():
    return [(t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1) for t in range(27)]


def im2col(x, dims):
    Z, Y, X = dims
    C = x.shape[1]
    g = x.reshape(Z, Y, X, C)
    pad = np.zeros((Z + 2, Y + 2, X + 2, C))
    pad[1:-1, 1:-1, 1:-1] = g
    cols = [pad[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X] for dx, dy, dz in _taps()]
    return np.stack(cols, axis=3).reshape(Z * Y * X, 27 * C)


def col2im(dcol, dims, C):
    Z, Y, X = dims
    d = dcol.reshape(Z, Y, X, 27, C)
    pad = np.zeros((Z + 2, Y + 2, X + 2, C))
    for t, (dx, dy, dz) in enumerate(_taps()):
        pad[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X] += d[:, :, :, t]
    return pad[1:-1, 1:-1, 1:-1].reshape(Z * Y * X, C)


def pool2(x, dims):
    Z, Y, X = dims
    C = x.shape[1]
    return x.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(1, 3, 5)).reshape(-1, C)


def pool2_back(d, dims):
    Z, Y, X = dims
    C = d.shape[1]
    g = d.reshape(Z // 2, 1, Y // 2, 1, X // 2, 1, C) / 8.0
    return np.broadcast_to(g, (Z // 2, 2, Y // 2, 2, X // 2, 2, C)).reshape(-1, C)


def up2(x, dims):
    Z, Y, X = dims
    C = x.shape[1]
    g = x.reshape(Z // 2, 1, Y // 2, 1, X // 2, 1, C)
    return np.broadcast_to(g, (Z // 2, 2, Y // 2, 2, X // 2, 2, C)).reshape(-1, C)


def up2_back(d, dims):
    Z, Y, X = dims
    C = d.shape[1]
    return d.reshape(Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(1, 3, 5)).reshape(-1, C)


def bf16(a):
    """Round to the nearest bf16 value (ties to even), returned as float64."""
    f = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((f + 0x7FFF + ((f >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_backward(params, x, dims, target, mask, quant=None):
    """Loss and gradients {name: (dW, db)} of the network for one case (float64).  `quant`
    (e.g. bf16) is applied wherever the GPU path stores a value in 16 bits: every layer's
    output but the last, the pooled and upsampled activations, and each layer's output
    gradient before its two gradient products."""
    q = quant or (lambda a: a)
    Z, Y, X = dims
    half = (Z // 2, Y // 2, X // 2)
    n = max(float(mask.sum()), 1.0)
    cache = {}

    def conv(name, inp, d, relu):
        W, b = params[name]
        col = im2col(inp, d)
        pre = col @ W.T + b
        out = np.maximum(pre, 0) if relu else pre
        if name != "c6":
            out = q(out)
        cache[name] = (col, out, d, relu, inp.shape[1])
        return out

    a1 = conv("c1", x, dims, True)
    p = q(pool2(a1, dims))
    a2 = conv("c2", p, half, True)
    a3 = conv("c3", a2, half, True)
    a4 = conv("c4", a3, half, True)
    u = q(up2(a4, dims) + a1)
    a5 = conv("c5", u, dims, True)
    out = conv("c6", a5, dims, False)
    diff = out[:, :4] - target
    loss = float((mask[:, None] * diff ** 2).sum() / n)
    dout = np.zeros_like(out)
    dout[:, :4] = 2 * mask[:, None] * diff / n

    grads = {}

    def conv_back(name, dy):
        col, y, d, relu, cin = cache[name]
        W, _ = params[name]
        g = dy * (y > 0) if relu else dy
        db = g.sum(0)
        g = q(g)
        grads[name] = (g.T @ col, db)
        return col2im(g @ W, d, cin)

    d5 = conv_back("c6", dout)
    du = conv_back("c5", d5)
    d4 = up2_back(du, dims)
    d3 = conv_back("c4", d4)
    d2 = conv_back("c3", d3)
    dp = conv_back("c2", d2)
    da1 = du + pool2_back(dp, dims)
    conv_back("c1", da1)
    return loss, out, grads
