"""ORACLE / TEST INFRASTRUCTURE ONLY.

CPU restatement of the learned drop-tolerance model: per-row features and
the 32 -> 64 -> 64 -> 2 MLP's forward and backward passes, in numpy, with
the same BF16 rounding points as the GPU kernels (round to nearest even):
x, W1, W2, W3 and the layer-1 activations are BF16; layer-2 activations stay
unrounded for layer 3; the layer-2 and layer-1 activation gradients are
rounded where they feed dH1 = dH2 W2, dW2 = dH2^T H1 and dW1 = dH1^T X,
and kept unrounded for the bias gradients and dW3.  Accumulation is FP64
here (FP32 on the GPU).  With rounding switched off the same code is the
plain FP64 network, which the tests check against finite differences.

The reference has no learned component; the model replaces the drop
tolerance search of fastainv/droptol-tuning.h:4-103.  Only tests/ import
this module.
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT = 32, 64, 2
W1, B1 = 0, N_H * N_IN
W2 = B1 + N_H
B2 = W2 + N_H * N_H
W3 = B2 + N_H
B3 = W3 + N_OUT * N_H
N_PARAMS = B3 + N_OUT


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even); returns float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def bf16_bits(x):
    """BF16 bit patterns (uint16) of float32 values, rounded like bf16()."""
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(b):
    return (np.asarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def unpack(params):
    p = np.asarray(params, np.float64)
    return (p[W1:B1].reshape(N_H, N_IN), p[B1:W2], p[W2:B2].reshape(N_H, N_H), p[B2:W3],
            p[W3:B3].reshape(N_OUT, N_H), p[B3:N_PARAMS])


def forward_backward(params, X, T=None, Wt=None, rounding=True):
    """X: [M, 32] features (BF16 values as float32); T, Wt: [M, 2] targets and
    weights.  Returns (Y, loss, grad) -- loss and grad None without T.
    Loss = sum_r sum_o w_ro (y_ro - t_ro)^2 / M."""
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(params)
    f32 = lambda a: np.asarray(a, np.float32)
    w1b, w2b, w3b = (np.asarray(r(f32(w) if rounding else w), np.float64) for w in (w1, w2, w3))
    Xb = np.asarray(r(f32(X)) if rounding else X, np.float64)
    h1p = Xb @ w1b.T + b1
    h1 = np.maximum(h1p, 0.0)
    h1b = np.asarray(r(f32(h1)) if rounding else h1, np.float64)
    h2p = h1b @ w2b.T + b2
    h2 = np.maximum(h2p, 0.0)
    Y = h2 @ w3b.T + b3
    if T is None:
        return Y, None, None
    M = X.shape[0]
    Wt = np.ones_like(T) if Wt is None else Wt
    e = Y - T
    loss = float(np.sum(Wt * e * e) / M)
    dY = 2.0 * Wt * e / M
    gW3 = dY.T @ h2
    gb3 = dY.sum(0)
    dH2 = (dY @ w3b) * (h2p > 0)
    gb2 = dH2.sum(0)
    dH2b = np.asarray(r(f32(dH2)) if rounding else dH2, np.float64)
    dH1 = (dH2b @ w2b) * (h1b > 0)
    gb1 = dH1.sum(0)
    dH1b = np.asarray(r(f32(dH1)) if rounding else dH1, np.float64)
    gW2 = dH2b.T @ h1b
    gW1 = dH1b.T @ Xb
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return Y, loss, grad


def row_features(row_ptr, cols, vals, nx=0, ny=0):
    """[n, 32] float32 features of an FP64 CSR (the layout of
    ispm_row_features); the GPU stores them as BF16."""
    n = len(row_ptr) - 1
    F = np.zeros((n, 32), np.float32)
    plane = nx * ny
    for i in range(n):
        lo, hi = row_ptr[i], row_ptr[i + 1]
        c, v = cols[lo:hi], vals[lo:hi]
        dm = c == i
        aii = float(v[dm][0]) if dm.any() else 0.0
        d = aii if aii > 0 else 1.0
        off = np.abs(v[~dm])
        nz = off[off > 0]
        f = np.zeros(32)
        f[0] = np.log(d) / 8.0
        f[1] = nz.sum() / d
        pos = 0
        for j, a in zip(c, v):
            if j == i:
                continue
            k = -1
            if nx > 0:
                dd = int(j) - i
                s = dd + plane + nx + 1
                dz = s // plane - 1 if s >= 0 else -2
                rem = dd - dz * plane
                s2 = rem + nx + 1
                dy = s2 // nx - 1 if s2 >= 0 else -2
                dx = rem - dy * nx
                if -1 <= dz <= 1 and -1 <= dy <= 1 and -1 <= dx <= 1:
                    q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)
                    k = q if q < 13 else q - 1
            elif pos < 26:
                k = pos
            pos += 1
            if k >= 0:
                f[2 + k] = abs(a) / d
        f[28] = 1.0 if hi - lo > 7 else 0.0
        f[29] = np.log(nz.max() / nz.min()) / 8.0 if nz.size >= 2 else 0.0
        f[30] = (hi - lo) / 27.0
        f[31] = 1.0
        F[i] = f.astype(np.float32)
    return F
