"""Test infrastructure (the oracle): numpy restatement of the warm-start
network's forward and backward passes (the kernels of csrc/mpnn.cu), used only
by tests to check the CUDA path.

``bf16=True`` rounds both operands of every matrix product to bfloat16
(round to nearest even), as the tensor-core kernels stage them; products are
accumulated in float64 here (float32 on the GPU). ``bf16=False`` is plain
float64 arithmetic, the version the finite-difference tests pin.
"""
from __future__ import annotations

import numpy as np


def to_bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unflatten(flat, width=128, layers=3, out=5, node_in=4, edge_in=3):
    shapes = [("Win", (node_in, width)), ("bin", (width,))]
    for l in range(layers):
        shapes += [(f"Wm{l}", (width + edge_in, width)), (f"bm{l}", (width,)),
                   (f"Wu{l}", (2 * width, width)), (f"bu{l}", (width,))]
    shapes += [("Wo", (width, out)), ("bo", (out,))]
    p, o = {}, 0
    for name, shape in shapes:
        size = int(np.prod(shape))
        p[name] = np.asarray(flat[o:o + size], dtype=np.float64).reshape(shape)
        o += size
    assert o == len(flat)
    return p, [name for name, _ in shapes]


def _mm(a, b, bf16):
    if bf16:
        a, b = to_bf16(a), to_bf16(b)
    return np.asarray(a, dtype=np.float64) @ np.asarray(b, dtype=np.float64)


def forward(p, layers, g, bf16=True):
    """g: dict(node [N, 4], src [E], dst [E], ef [E, 3]). Returns (theta, cache)."""
    node, src, dst, ef = g["node"], g["src"], g["dst"], g["ef"]
    N = node.shape[0]
    deg = np.bincount(dst, minlength=N).astype(np.float64)
    X = [np.maximum(_mm(node, p["Win"], bf16) + p["bin"], 0.0)]
    Ms, As, Rs = [], [], []
    for l in range(layers):
        inp = np.concatenate([X[l][src], ef], axis=1)
        M = np.maximum(_mm(inp, p[f"Wm{l}"], bf16) + p[f"bm{l}"], 0.0)
        A = np.zeros_like(X[l])
        np.add.at(A, dst, M)
        A = np.where(deg[:, None] > 0, A / np.maximum(deg, 1)[:, None], 0.0)
        R = np.maximum(_mm(np.concatenate([X[l], A], axis=1), p[f"Wu{l}"], bf16) + p[f"bu{l}"], 0.0)
        X.append(X[l] + R)
        Ms.append(M)
        As.append(A)
        Rs.append(R)
    Z = _mm(X[layers], p["Wo"], bf16) + p["bo"]
    theta = np.pi * np.tanh(Z)
    return theta, dict(X=X, M=Ms, A=As, R=Rs, Z=Z, deg=deg)


def backward(p, layers, g, cache, dtheta, bf16=True):
    """Gradients (dict by parameter name) of sum(dtheta * theta)."""
    node, src, dst, ef = g["node"], g["src"], g["dst"], g["ef"]
    X, Ms, As, Rs, Z, deg = cache["X"], cache["M"], cache["A"], cache["R"], cache["Z"], cache["deg"]
    grads = {}
    dZ = dtheta * np.pi * (1.0 - np.tanh(Z) ** 2)
    grads["Wo"] = _mm(X[layers].T, dZ, bf16)
    grads["bo"] = dZ.sum(0)
    dX = _mm(dZ, p["Wo"].T, bf16)
    W = X[0].shape[1]
    for l in range(layers - 1, -1, -1):
        dU = dX * (Rs[l] > 0)
        cat = np.concatenate([X[l], As[l]], axis=1)
        grads[f"Wu{l}"] = _mm(cat.T, dU, bf16)
        grads[f"bu{l}"] = dU.sum(0)
        G = _mm(dU, p[f"Wu{l}"].T, bf16)
        dX = dX + G[:, :W]
        dA = G[:, W:]
        dV = (dA[dst] / deg[dst][:, None]) * (Ms[l] > 0)
        inp = np.concatenate([X[l][src], ef], axis=1)
        grads[f"Wm{l}"] = _mm(inp.T, dV, bf16)
        grads[f"bm{l}"] = dV.sum(0)
        S = np.zeros_like(X[l])
        np.add.at(S, src, dV)
        dX = dX + _mm(S, p[f"Wm{l}"][:W].T, bf16)
    dpre = dX * (X[0] > 0)
    grads["Win"] = _mm(node.T, dpre, bf16)
    grads["bin"] = dpre.sum(0)
    return grads


def flatten(grads, names):
    return np.concatenate([np.asarray(grads[n], dtype=np.float64).reshape(-1) for n in names])


def periodic_loss(theta, target, weight=None):
    """(loss, dloss/dtheta) of sum_i w_i sum_j (1 - cos(theta - target)) / (out * sum w)."""
    N, out = theta.shape
    w = np.ones(N) if weight is None else np.asarray(weight, dtype=np.float64)
    scale = 1.0 / (w.sum() * out)
    d = theta - target
    return float((w[:, None] * (1 - np.cos(d))).sum() * scale), w[:, None] * np.sin(d) * scale


def adam(w, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    g = g + wd * w
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v
