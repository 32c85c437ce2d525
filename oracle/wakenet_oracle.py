"""CPU oracle of the wake network (test infrastructure only).

A float64 NumPy restatement of the network that elegant_b200/csrc/b2e_wakenet.cu
trains on the tensor cores: 6 dilated 1-D convolutions (64 channels, 5 taps,
zero padding), GELU (erf form) after the first five, output channel 0 of the
last, mean-squared-error loss, and its exact backward pass.  With bf16=True
the values are rounded to BF16 exactly where the device kernels store BF16
(input pack, weights, pre-activations, activations, back-propagated
gradients); with bf16=False everything stays float64, which is what the
finite-difference check of the backward pass uses.

The network has no counterpart in the reference; the data it is trained on
(the wake integral) is pinned separately against the reference's csbend.c.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

LAYERS, CH, TAPS = 6, 64, 5
WSIZE = TAPS * CH * CH
NPARAM = LAYERS * (WSIZE + CH)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def split(params: np.ndarray):
    w = params[: LAYERS * WSIZE].reshape(LAYERS, TAPS, CH, CH)  # [l][t][co][ci]
    b = params[LAYERS * WSIZE:].reshape(LAYERS, CH)
    return w, b


def gelu(z):
    return 0.5 * z * (1 + erf(z / np.sqrt(2)))


def gelu_grad(z):
    return 0.5 * (1 + erf(z / np.sqrt(2))) + z * np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)


def _shift(x: np.ndarray, k: int) -> np.ndarray:
    """out[:, i] = x[:, i + k], zero outside [0, L)."""
    out = np.zeros_like(x)
    L = x.shape[1]
    if k >= 0:
        if k < L:
            out[:, : L - k] = x[:, k:]
    else:
        if -k < L:
            out[:, -k:] = x[:, : L + k]
    return out


def conv(x, w, d, sign=1):
    """x [n][L][64], w [5][co][ci] -> [n][L][co]; tap t reads bin i + sign*(t-2)*d."""
    out = np.zeros(x.shape[:2] + (w.shape[1],))
    for t in range(TAPS):
        out += _shift(x, sign * (t - 2) * d) @ w[t].T
    return out


def conv_t(g, w, d):
    """Transposed convolution: g [n][L][co] -> [n][L][ci]."""
    out = np.zeros(g.shape[:2] + (w.shape[2],))
    for t in range(TAPS):
        out += _shift(g, -(t - 2) * d) @ w[t]
    return out


def pack(inputs: np.ndarray, use_bf16: bool) -> np.ndarray:
    """inputs [n][c][L] -> [n][L][64] with channels c..63 zero."""
    n, c, L = inputs.shape
    x = np.zeros((n, L, CH))
    x[:, :, :c] = np.transpose(inputs, (0, 2, 1))
    return bf16(x) if use_bf16 else x


def forward(params, inputs, dilations, use_bf16=True):
    w, b = split(np.asarray(params, dtype=np.float64))
    if use_bf16:
        w = bf16(w)
    x = pack(np.asarray(inputs, dtype=np.float64), use_bf16)
    xs, zs = [x], []
    for l in range(LAYERS - 1):
        z = conv(xs[-1], w[l], dilations[l]) + b[l]
        a = gelu(z)
        zs.append(bf16(z) if use_bf16 else z)
        xs.append(bf16(a) if use_bf16 else a)
    y = conv(xs[-1], w[-1][:, :1, :], dilations[-1])[:, :, 0] + b[-1][0]
    return y, (w, xs, zs)


def loss_and_gradients(params, inputs, targets, dilations, use_bf16=True):
    """Mean squared error and its gradient with respect to the flat parameters."""
    y, (w, xs, zs) = forward(params, inputs, dilations, use_bf16)
    r = y - np.asarray(targets, dtype=np.float64)
    rows = r.size
    loss = float((r * r).sum() / rows)
    dz = np.zeros(y.shape + (CH,))
    dz[:, :, 0] = bf16(r) if use_bf16 else r
    scale = 2.0 / rows
    gw = np.zeros((LAYERS, TAPS, CH, CH))
    gb = np.zeros((LAYERS, CH))
    for l in range(LAYERS - 1, -1, -1):
        x, d = xs[l], dilations[l]
        flat_dz = dz.reshape(-1, CH)
        for t in range(TAPS):
            gw[l, t] = scale * flat_dz.T @ _shift(x, (t - 2) * d).reshape(-1, CH)
        gb[l] = scale * flat_dz.sum(axis=0)
        if l > 0:
            da = conv_t(dz, w[l], d)
            g = da * gelu_grad(zs[l - 1])
            dz = bf16(g) if use_bf16 else g
    return loss, np.concatenate([gw.ravel(), gb.ravel()])
