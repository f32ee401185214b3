"""TEST INFRASTRUCTURE ONLY: numpy restatement of the learned U-Net
preconditioner (forward, backward, Adam), the checker of the library's
tcgen05 kernels.  It has no counterpart in the reference (the learned
preconditioner is new in this implementation); its arithmetic is the
textbook one: 3x3x3 convolutions (periodic in x and y, zero outside z),
ReLU, 2x2x2 mean pooling, nearest upsampling, additive skips.

Tensors are channels-last float arrays (nz, ny, nx, C).  Activations and
weights pass through bfloat16 (round to nearest even) where the GPU stores
them in bfloat16; sums are float64 here (the GPU accumulates in float32).

Network (levels 16/32/32 channels):
    x (2 ch: r s with unit RMS on the fluid, fluid mask) padded to 16 channels
    e1a = relu(conv(x, 16->16));      e1 = relu(conv(e1a, 16->16))
    p1  = pool(e1)
    e2a = relu(conv(p1, 16->32));     e2 = relu(conv(e2a, 32->32))
    p2  = pool(e2)
    e3a = relu(conv(p2, 32->32));     e3 = relu(conv(e3a, 32->32))
    u2  = up(e3) + e2
    d2  = relu(conv(u2, 32->16))
    u1  = up(d2) + e1
    d1  = relu(conv(u1, 16->16))
    out = conv(d1, 16->16)[..., 0]    (one output channel of a padded layer)
"""
from __future__ import annotations

import numpy as np

LAYERS = (("e1a", 16, 16), ("e1", 16, 16), ("e2a", 16, 32), ("e2", 32, 32), ("e3a", 32, 32), ("e3", 32, 32),
          ("d2", 32, 16), ("d1", 16, 16), ("out", 16, 16))


def bf16(a):
    """Round float values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def bf16_bits(a):
    a = bf16(a)
    return (a.view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(u):
    return (np.asarray(u, dtype=np.uint32) << 16).view(np.float32)


def taps():
    """(dz, dy, dx) of tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)."""
    return [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def shift(x, dz, dy, dx):
    """y[z, j, i] = x[z+dz, (j+dy)%ny, (i+dx)%nx] (zero outside z)."""
    y = np.roll(x, (-dy, -dx), axis=(1, 2))
    out = np.zeros_like(y)
    nz = x.shape[0]
    if dz == 0:
        out[:] = y
    elif dz == 1:
        out[:nz - 1] = y[1:]
    else:
        out[1:] = y[:nz - 1]
    return out


def conv(x, W, b):
    """out[z,y,x,co] = b[co] + sum_t sum_ci x[nbr_t, ci] W[t, co, ci]."""
    nz, ny, nx, ci = x.shape
    co = W.shape[1]
    acc = np.zeros((nz, ny, nx, co), dtype=np.float64) + b.astype(np.float64)
    for t, (dz, dy, dx) in enumerate(taps()):
        acc += shift(x, dz, dy, dx).astype(np.float64) @ W[t].T.astype(np.float64)
    return acc


def conv_backward(x, W, g):
    """Gradients of conv: (dx, dW, db) for the output gradient g."""
    dx = np.zeros(x.shape, dtype=np.float64)
    dW = np.zeros(W.shape, dtype=np.float64)
    for t, (dz, dy, dxs) in enumerate(taps()):
        xs = shift(x, dz, dy, dxs).astype(np.float64)
        dW[t] = np.einsum("zyxo,zyxi->oi", g, xs)
        dx += shift(g @ W[t].astype(np.float64), -dz, -dy, -dxs)
    return dx, dW, g.sum(axis=(0, 1, 2))


def pool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def pool_backward(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)


def up_backward(g):
    nz, ny, nx, c = g.shape
    return g.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).sum(axis=(1, 3, 5))


def init_params(seed=0):
    """He-normal weights (std sqrt(2 / (27 ci))), zero biases; the last
    layer's padded output channels are zero."""
    rng = np.random.default_rng(seed)
    P = {}
    for name, ci, co in LAYERS:
        std = np.sqrt(2.0 / (27 * ci)) * (0.1 if name == "out" else 1.0)
        W = rng.standard_normal((27, co, ci)) * std
        if name == "e1a":
            W[:, :, 2:] = 0.0
        if name == "out":
            W[:, 1:, :] = 0.0
        P[name] = (W.astype(np.float32), np.zeros(co, dtype=np.float32))
    return P


def input_scale(r, mask):
    """s = sqrt(n_fluid / sum over fluid of r^2): r s has unit RMS on the fluid."""
    f = mask > 0
    ss = float((r[f].astype(np.float64) ** 2).sum())
    return np.sqrt(f.sum() / ss) if ss > 0 else 1.0


def inputs(r, mask):
    """The 16-channel input: r s, the fluid mask, zeros."""
    nz, ny, nx = r.shape
    x = np.zeros((nz, ny, nx, 16), dtype=np.float32)
    x[..., 0] = (r * np.float32(input_scale(r, mask))).astype(np.float32)
    x[..., 1] = mask
    return bf16(x)


def forward(P, x):
    """Activations of every layer (bf16-rounded where the GPU stores bf16)."""
    A = {"x": x}

    def layer(name, inp, relu=True, add=None):
        W, b = P[name]
        y = conv(inp, bf16(W), b)
        if add is not None:
            y = y + add
        if relu:
            y = np.maximum(y, 0.0)
        return y

    A["e1a"] = bf16(layer("e1a", x))
    A["e1"] = bf16(layer("e1", A["e1a"]))
    A["p1"] = bf16(pool(A["e1"]))
    A["e2a"] = bf16(layer("e2a", A["p1"]))
    A["e2"] = bf16(layer("e2", A["e2a"]))
    A["p2"] = bf16(pool(A["e2"]))
    A["e3a"] = bf16(layer("e3a", A["p2"]))
    A["e3"] = bf16(layer("e3", A["e3a"]))
    A["u2"] = bf16(up(A["e3"]) + A["e2"])
    A["d2"] = bf16(layer("d2", A["u2"]))
    A["u1"] = bf16(up(A["d2"]) + A["e1"])
    A["d1"] = bf16(layer("d1", A["u1"]))
    A["out"] = layer("out", A["d1"], relu=False)[..., 0]
    return A


def loss_and_grad_out(out, target, mask):
    """L = sum over fluid cells of (z - mean z - (e - mean e))^2 / n_fluid,
    z the raw output, e the error scaled to unit RMS on the fluid; returns
    (L, dL/dz)."""
    f = mask > 0
    target = target * np.sqrt(f.sum() / (target[f].astype(np.float64) ** 2).sum())
    nf = max(int(f.sum()), 1)
    z = np.where(f, out, 0.0)
    e = np.where(f, target, 0.0)
    d = (z - z[f].mean()) - (e - e[f].mean())
    d = np.where(f, d, 0.0)
    L = float((d[f] ** 2).sum() / nf)
    g = 2.0 * d / nf
    g = np.where(f, g - g[f].mean(), 0.0)
    return L, g


def backward(P, A, gout):
    """Parameter gradients {name: (dW, db)} for the output gradient gout."""
    G = {}

    def relu_grad(g, y):
        return np.where(y > 0, g, 0.0)

    g = np.zeros(A["d1"].shape[:3] + (16,))
    g[..., 0] = gout
    gx, dW, db = conv_backward(A["d1"], bf16(P["out"][0]), g)
    G["out"] = (dW, db)
    g = relu_grad(gx, A["d1"])
    gx, dW, db = conv_backward(A["u1"], bf16(P["d1"][0]), g)
    G["d1"] = (dW, db)
    g_e1 = gx.copy()
    g = relu_grad(up_backward(gx), A["d2"])
    gx, dW, db = conv_backward(A["u2"], bf16(P["d2"][0]), g)
    G["d2"] = (dW, db)
    g_e2 = gx.copy()
    g = relu_grad(up_backward(gx), A["e3"])
    gx, dW, db = conv_backward(A["e3a"], bf16(P["e3"][0]), g)
    G["e3"] = (dW, db)
    g = relu_grad(gx, A["e3a"])
    gx, dW, db = conv_backward(A["p2"], bf16(P["e3a"][0]), g)
    G["e3a"] = (dW, db)
    g = relu_grad(g_e2 + pool_backward(gx), A["e2"])
    gx, dW, db = conv_backward(A["e2a"], bf16(P["e2"][0]), g)
    G["e2"] = (dW, db)
    g = relu_grad(gx, A["e2a"])
    gx, dW, db = conv_backward(A["p1"], bf16(P["e2a"][0]), g)
    G["e2a"] = (dW, db)
    g = relu_grad(g_e1 + pool_backward(gx), A["e1"])
    gx, dW, db = conv_backward(A["e1a"], bf16(P["e1"][0]), g)
    G["e1"] = (dW, db)
    g = relu_grad(gx, A["e1a"])
    _, dW, db = conv_backward(A["x"], bf16(P["e1a"][0]), g)
    G["e1a"] = (dW, db)
    return G


def adam(P, G, M, V, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the FP32 master weights (Kingma & Ba 2015)."""
    out = {}
    for name, _, _ in LAYERS:
        newp = []
        for q in range(2):
            p, g = P[name][q].astype(np.float64), G[name][q]
            M[name][q] = b1 * M[name][q] + (1 - b1) * g
            V[name][q] = b2 * V[name][q] + (1 - b2) * g * g
            mh = M[name][q] / (1 - b1 ** step)
            vh = V[name][q] / (1 - b2 ** step)
            newp.append((p - lr * mh / (np.sqrt(vh) + eps)).astype(np.float32))
        out[name] = tuple(newp)
    return out
