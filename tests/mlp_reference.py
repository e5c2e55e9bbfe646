"""CPU restatement of the warm-start network, for checking the tensor-core
kernels: same features, same BF16 rounding points (inputs, weights, and each
hidden activation before it enters the next GEMM; dZ before the backward
GEMMs), FP32/FP64 accumulation."""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SHAPES = [("w1", "b1", 64, 32), ("w2", "b2", 64, 64), ("w3", "b3", 64, 64), ("w4", "b4", 32, 64)]


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def features(image: np.ndarray) -> np.ndarray:
    h, w, _ = image.shape
    f = np.zeros((h * w, 32), np.float32)
    k = 0
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            yy = np.clip(np.arange(h)[:, None] + dy, 0, h - 1)
            xx = np.clip(np.arange(w)[None, :] + dx, 0, w - 1)
            f[:, k:k + 3] = image[yy, xx].reshape(-1, 3)
            k += 3
    f[:, 27:30] = np.log(image.reshape(-1, 3).astype(np.float32) + np.float32(1 / 256))
    return f


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def params(model):
    return [(bf16(model.get(w)).astype(np.float64), model.get(b).astype(np.float64)) for w, b, _, _ in SHAPES]


def forward(model, feats, round_hidden=True):
    P = params(model)
    h = bf16(feats).astype(np.float64)
    hs, zs = [h], []
    for k, (W, b) in enumerate(P):
        z = h @ W.T + b
        zs.append(z)
        if k < 3:
            h = gelu(z)
            h = bf16(h).astype(np.float64) if round_hidden else h
            hs.append(h)
    y = 1.0 / (1.0 + np.exp(-zs[-1]))
    return y, hs, zs


def loss_grad(model, feats, targets, round_hidden=True):
    """Mean squared error over samples and outputs, and its gradients."""
    n, outs = targets.shape
    P = params(model)
    y, hs, zs = forward(model, feats, round_hidden)
    e = y[:, :outs] - targets
    loss = float(np.mean(e * e))
    dz = np.zeros_like(y)
    dz[:, :outs] = 2.0 / (n * outs) * e * y[:, :outs] * (1 - y[:, :outs])
    grads = {}
    for k in (3, 2, 1, 0):
        dzr = bf16(dz).astype(np.float64) if round_hidden else dz
        grads[SHAPES[k][0]] = dzr.T @ hs[k]
        grads[SHAPES[k][1]] = dz.sum(axis=0)
        if k > 0:
            dh = dzr @ P[k][0]
            dz = dh * gelu_grad(zs[k - 1])
    return loss, grads
