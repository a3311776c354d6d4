"""ORACLE -- test infrastructure, not the product.

CPU (numpy, FP64) restatement of the learned pruning-radius model of ebgeometry_b200/csrc/seed.cu:
the 16-level hash-grid encoding and the 32-64-64-64-1 ReLU MLP, forward and backward, with the
product's BF16 rounding points reproduced (forward: table entries, encoding, weights and hidden
activations; backward: the layer deltas where they enter the weight- and input-gradient products as
tensor-core operands) and everything else in FP64.  The model has no counterpart
in the reference; this restatement is what the GPU gradients are checked against.
"""
from __future__ import annotations

import numpy as np

LEVELS, FEATS, IN, WIDTH = 16, 2, 32, 64
W1, B1 = 0, 64 * 32
W2, B2 = B1 + 64, B1 + 64 + 64 * 64
W3, B3 = B2 + 64, B2 + 64 + 64 * 64
W4, B4 = B3 + 64, B3 + 64 + 64
NPARAM = B4 + 1


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def levels(base, maxres, log2t):
    b = np.exp((np.log(maxres) - np.log(base)) / (LEVELS - 1))
    res = [int(np.floor(base * b ** l + 1e-9)) for l in range(LEVELS)]
    dense = [int((r + 1) ** 3 <= 2 ** log2t) for r in res]
    return res, dense


def corners(p, lo, scale, res, dense, log2t):
    """Per level: (indices (n,8) int64, weights (n,8))."""
    u = np.clip((p - lo) * scale, 0.0, 1.0)
    T = 1 << log2t
    out = []
    for l in range(LEVELS):
        N = res[l]
        x = u * N
        i0 = np.minimum(np.floor(x).astype(np.int64), N - 1)
        f = x - i0
        idx = np.zeros((p.shape[0], 8), np.int64)
        w = np.ones((p.shape[0], 8))
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, k >> 2])
            c = i0 + d
            for a in range(3):
                w[:, k] *= np.where(d[a] == 1, f[:, a], 1.0 - f[:, a])
            if dense[l]:
                r = N + 1
                idx[:, k] = (c[:, 2] * r + c[:, 1]) * r + c[:, 0]
            else:
                h = (c[:, 0].astype(np.uint64) ^ (c[:, 1].astype(np.uint64) * np.uint64(2654435761))
                     ^ (c[:, 2].astype(np.uint64) * np.uint64(805459861))) & np.uint64(0xFFFFFFFF)
                idx[:, k] = (h & np.uint64(T - 1)).astype(np.int64)
        out.append((idx, w))
    return out


def loss_and_grads(p, d, table, params, lo, scale, res, dense, log2t, eps):
    """loss = sum w (y - d)^2 / n, w = 1/(|d|+eps)^2; returns (loss, grad_table, grad_params, y)."""
    n = p.shape[0]
    T = 1 << log2t
    tab = bf16(table).reshape(LEVELS, T, 2)
    cs = corners(p.astype(np.float64), lo, scale, res, dense, log2t)
    X = np.zeros((n, IN))
    for l, (idx, w) in enumerate(cs):
        X[:, 2 * l] = (w * tab[l][idx, 0]).sum(1)
        X[:, 2 * l + 1] = (w * tab[l][idx, 1]).sum(1)
    Xb = bf16(X)
    P = params.astype(np.float64)
    w1 = bf16(P[W1:B1]).reshape(64, 32)
    w2 = bf16(P[W2:B2]).reshape(64, 64)
    w3 = bf16(P[W3:B3]).reshape(64, 64)
    w4 = bf16(P[W4:B4])
    b1, b2, b3, b4 = P[B1:W2], P[B2:W3], P[B3:W4], P[B4]
    H1 = bf16(np.maximum(Xb @ w1.T + b1, 0))
    H2 = bf16(np.maximum(H1 @ w2.T + b2, 0))
    H3 = bf16(np.maximum(H2 @ w3.T + b3, 0))
    y = H3 @ w4 + b4
    wt = 1.0 / (np.abs(d) + eps) ** 2
    loss = np.sum(wt * (y - d) ** 2) / n
    dy = 2 * wt * (y - d) / n
    g = np.zeros(NPARAM)
    # The device forms every gradient but b4 as a tensor-core product over the samples, with BF16
    # operands: the deltas and dy are rounded to BF16, and the bias gradients are products with a
    # row of ones (sums of the rounded deltas).  b4's gradient sums dy in FP32.
    g[W4:B4] = H3.T @ bf16(dy)
    g[B4] = dy.sum()
    dH3 = np.outer(dy, w4) * (H3 > 0)
    g[W3:B3] = (bf16(dH3).T @ H2).ravel()
    g[B3:W4] = bf16(dH3).sum(0)
    dH2 = (bf16(dH3) @ w3) * (H2 > 0)
    g[W2:B2] = (bf16(dH2).T @ H1).ravel()
    g[B2:W3] = bf16(dH2).sum(0)
    dH1 = (bf16(dH2) @ w2) * (H1 > 0)
    g[W1:B1] = (bf16(dH1).T @ Xb).ravel()
    g[B1:W2] = bf16(dH1).sum(0)
    dX = bf16(dH1) @ w1
    gt = np.zeros((LEVELS, T, 2))
    for l, (idx, w) in enumerate(cs):
        for f in range(2):
            np.add.at(gt[l, :, f], idx.ravel(), (w * dX[:, 2 * l + f][:, None]).ravel())
    return loss, gt.ravel(), g, y
