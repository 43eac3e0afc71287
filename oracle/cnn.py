"""CPU restatement of the learned early stop's network (test infrastructure).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA kernels of
ems_b200/csrc/learn.cu (forward, backward). numpy, float64 accumulation,
with the GEMM operands rounded to bf16 as the tensor-core kernels read them
(round to nearest even), so the only differences left are the order of f32
sums on the device. The network itself has no counterpart in the
reference; its layers are those described in ems_b200/learn.py.
"""
from __future__ import annotations

import numpy as np

from ems_b200.learn import CONVS, HIDDEN, layer_shapes, param_views


def bf16(x: np.ndarray) -> np.ndarray:
    """Round f32 values to bf16 (nearest even), returned as f64."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(y):
    return y / (1.0 + np.exp(-y))


def silu_grad(y):
    s = 1.0 / (1.0 + np.exp(-y))
    return s + y * s * (1.0 - s)


def im2col(x, k, s):
    """x (B, T, C) → (B·T_out, k·C), rows (b, t_out), columns (tap, channel)."""
    B, T, C = x.shape
    To = (T - k) // s + 1
    idx = np.arange(To)[:, None] * s + np.arange(k)[None, :]
    return x[:, idx, :].reshape(B * To, k * C)


def col2im(dcol, B, T, C, k, s):
    To = (T - k) // s + 1
    d = dcol.reshape(B, To, k, C)
    dx = np.zeros((B, T, C))
    for tap in range(k):
        dx[:, tap:tap + s * To:s, :] += d[:, :, tap, :]
    return dx


def forward(params, x, t_out, round_bf16=True):
    """Output (B, 2·t_out) and the cache for backward."""
    q = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    k_in = x.shape[1]
    W = param_views(np.asarray(params, dtype=np.float32 if round_bf16 else np.float64), k_in, t_out)
    B = x.shape[0]
    cache = {"x": [], "col": [], "y": []}
    a = np.asarray(x, dtype=np.float64)
    for l, (ci, co, k, s) in enumerate(CONVS):
        col = q(im2col(a, k, s))
        y = col @ q(W[l][0]).T + W[l][1]
        cache["x"].append(a)
        cache["col"].append(col)
        cache["y"].append(y)
        a = silu(y).reshape(B, -1, co)
    flat = q(a.reshape(B, -1))
    y4 = flat @ q(W[3][0]).T + W[3][1]
    a4 = q(silu(y4))
    out = a4 @ q(W[4][0]).T + W[4][1]
    cache.update(flat=flat, y4=y4, a4=a4, W=W, B=B, k_in=k_in)
    return out, cache


def backward(cache, dout, t_out, round_bf16=True):
    """Flat gradient (the layout of the parameters) of Σ dout·out."""
    q = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W, B, k_in = cache["W"], cache["B"], cache["k_in"]
    _, T = layer_shapes(k_in, t_out)
    grads = [None] * 5
    dy5 = np.asarray(dout, dtype=np.float64)
    dy5q = q(dy5)
    grads[4] = (dy5q.T @ cache["a4"], dy5.sum(axis=0))
    da4 = dy5q @ q(W[4][0])
    dy4 = da4 * silu_grad(cache["y4"])
    dy4q = q(dy4)
    grads[3] = (dy4q.T @ cache["flat"], dy4.sum(axis=0))
    da = dy4q @ q(W[3][0])
    for l in range(len(CONVS) - 1, -1, -1):
        ci, co, k, s = CONVS[l]
        dy = da.reshape(-1, co) * silu_grad(cache["y"][l])
        dyq = q(dy)
        grads[l] = (dyq.T @ cache["col"][l], dy.sum(axis=0))
        if l == 0:
            break
        dcol = dyq @ q(W[l][0])
        da = col2im(dcol, B, T[l], ci, k, s)
    return np.concatenate([np.concatenate([g[0].ravel(), g[1].ravel()]) for g in grads])
