"""CPU oracle of the proposer MLP (TEST INFRASTRUCTURE, checker only).

Forward and backward of the network libkls.so trains (kls_mlp_*):
5 -> width (GELU) -> ... -> 3, mean-squared-error loss, flat parameter order
W_l [out][in] then b_l [out] per layer.  With ``bf16=True`` operands are
rounded to BF16 exactly where the device rounds them (GEMM inputs: features,
activations, weights, output gradients), everything else in FP32, products
accumulated in FP64; with ``bf16=False`` the computation is plain FP64 (used
for a finite-difference check of the backward pass itself).
"""
from __future__ import annotations

import numpy as np
import scipy.special as sps


def bf16(x):
    """Round to BF16 (nearest even) and return as float32."""
    x = np.asarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def layer_shapes(width: int, depth: int):
    return [(5 if l == 0 else width, 3 if l == depth - 1 else width) for l in range(depth)]


def unpack(params: np.ndarray, width: int, depth: int):
    Ws, bs, o = [], [], 0
    for di, do in layer_shapes(width, depth):
        Ws.append(params[o:o + di * do].reshape(do, di)); o += di * do
        bs.append(params[o:o + do]); o += do
    return Ws, bs


def gelu(x):
    return 0.5 * x * (1.0 + sps.erf(x / np.sqrt(2.0)))


def gelu_d(x):
    return 0.5 * (1.0 + sps.erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


def forward_backward(params, X, T, width, depth, bf16_ops=True):
    """Returns (Y, loss, grads) with grads in the flat parameter order."""
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, dtype=np.float64))
    f = (lambda a: np.asarray(a, dtype=np.float32)) if bf16_ops else \
        (lambda a: np.asarray(a, dtype=np.float64))
    Ws, bs = unpack(np.asarray(params, dtype=np.float64 if not bf16_ops else np.float32),
                    width, depth)
    H = [r(X)]
    Z = []
    for l in range(depth):
        z = f(H[-1].astype(np.float64) @ r(Ws[l]).astype(np.float64).T) + f(bs[l])
        Z.append(f(z))
        if l < depth - 1:
            H.append(r(f(gelu(Z[-1].astype(np.float64)))))
    Y = Z[-1]
    B = X.shape[0]
    d = Y.astype(np.float64) - T
    loss = float(np.mean(d * d))
    dZ = f(2.0 * d / (B * 3))
    gW, gb = [None] * depth, [None] * depth
    for l in range(depth - 1, -1, -1):
        dZr = r(dZ)
        gW[l] = f(dZr.astype(np.float64).T @ H[l].astype(np.float64))
        gb[l] = f(np.sum(dZ.astype(np.float64), axis=0))
        if l == 0:
            break
        dH = f(dZr.astype(np.float64) @ r(Ws[l]).astype(np.float64))
        dZ = f(dH.astype(np.float64) * gelu_d(Z[l - 1].astype(np.float64)))
    grads = np.concatenate([np.concatenate([gW[l].ravel(), gb[l].ravel()]) for l in range(depth)])
    return Y, loss, grads
