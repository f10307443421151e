"""FP64 numpy reference of the residual CNN (forward and backward).

TEST INFRASTRUCTURE ONLY: the checker for the GPU CNN kernels' gradients.
Same layer table, padding (zero, "same") and parameter layout as the
library: input packing (pack_input); per layer weights [9 taps][cout][cin] (tap = ky*3 + kx, offset
((ky-1) d, (kx-1) d) for the layer's dilation d) then biases [cout];
loss = sum((out - target)^2) / (3 n).
"""
from __future__ import annotations

import numpy as np

LAYERS = [(7, 48)] + [(48, 48)] * 6 + [(48, 3)]
DILATIONS = [1, 2, 3, 4, 3, 2, 1, 1]


def unpack(params):
    out, o = [], 0
    for cin, cout in LAYERS:
        nw = 9 * cout * cin
        out.append((params[o:o + nw].reshape(9, cout, cin), params[o + nw:o + nw + cout]))
        o += nw + cout
    return out


def conv(x, w, b, d=1):
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (d, d), (d, d), (0, 0)))
    out = np.zeros((B, H, W, w.shape[1]))
    for t in range(9):
        ky, kx = divmod(t, 3)
        out += xp[:, ky * d:ky * d + H, kx * d:kx * d + W, :] @ w[t].T
    return out + b


def conv_back(x, w, dy, d=1):
    """(dx, dw, db) of conv(x, w, b, d) given dy."""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (d, d), (d, d), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for t in range(9):
        ky, kx = divmod(t, 3)
        xs = xp[:, ky * d:ky * d + H, kx * d:kx * d + W, :]
        dw[t] = np.einsum("bhwo,bhwi->oi", dy, xs)
        dxp[:, ky * d:ky * d + H, kx * d:kx * d + W, :] += dy @ w[t]
    return dxp[:, d:H + d, d:W + d, :], dw, dy.sum(axis=(0, 1, 2))


def pack_input(rgb, strength):
    """The network's input [B, H, W, 7] from float32 RGB [B, H, W, 3] and a
    strength (scalar or [B, H, W] map), as the library forms it (float32):
    channels 0-2 the RGB minus its 3x3 local mean (clamped edges; summed row
    by row, then / 9), 3-5 that mean, 6 the strength."""
    rgb = np.asarray(rgb, np.float32)
    B, H, W, _ = rgb.shape
    pad = np.pad(rgb, ((0, 0), (1, 1), (1, 1), (0, 0)), mode="edge")
    m = np.zeros_like(rgb)
    for dy in range(3):
        for dx in range(3):
            m = m + pad[:, dy:dy + H, dx:dx + W, :]
    m = m / np.float32(9)
    smap = np.broadcast_to(np.asarray(strength, np.float32)[..., None], rgb.shape[:3] + (1,))
    return np.concatenate([rgb - m, m, smap], axis=-1).astype(np.float32)


def forward(params, x, rgb):
    """out = rgb + network(x) for a packed input x [B, H, W, 7] (pack_input)."""
    layers = unpack(np.asarray(params, np.float64))
    x = np.asarray(x, np.float64)
    rgb = np.asarray(rgb, np.float64)
    acts = [x]
    for i, (w, b) in enumerate(layers):
        y = conv(acts[-1], w, b, DILATIONS[i])
        acts.append(np.maximum(y, 0) if i < len(layers) - 1 else y)
    return rgb + acts[-1], acts


def gradients(params, x, rgb, target, weight=None):
    """(flat gradient, loss_sum) of sum(weight * (out - target)^2) / (3 n) for
    out = forward(params, x, rgb); weight: None (1), a scalar or a [B, H, W] map."""
    layers = unpack(np.asarray(params, np.float64))
    out, acts = forward(params, x, rgb)
    n = rgb.shape[0] * rgb.shape[1] * rgb.shape[2]
    d = out - target
    wt = 1.0 if weight is None else np.broadcast_to(np.asarray(weight, np.float64)[..., None], d.shape)
    dy = 2.0 * wt * d / (3.0 * n)
    grads = []
    for i in range(len(layers) - 1, -1, -1):
        w, _ = layers[i]
        dx, dw, db = conv_back(acts[i], w, dy, DILATIONS[i])
        grads.append((dw, db))
        if i > 0:
            dy = dx * (acts[i] > 0)
    flat = []
    for dw, db in reversed(grads):
        flat += [dw.ravel(), db.ravel()]
    return np.concatenate(flat), float((wt * d ** 2).sum())


def bf16_round(a):
    """Round float32 values to bfloat16 (nearest-even) and back."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)
