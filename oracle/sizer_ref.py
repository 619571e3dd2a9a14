"""CPU reference of the learned sizer's network -- TEST INFRASTRUCTURE (the checker).

A 16 -> 64 -> 64 -> 1 multilayer perceptron with ReLU, weights stored in BF16 and every dot
product accumulated in FP32, regressing log2(1 + output nnz of a row).  The loss is the mean
squared error over a batch.  This module recomputes the forward pass and the exact gradients
with numpy so the CUDA kernels (partc_b200/csrc/ptc_sizer.cu) can be checked against it.

Parameter layout (the flat order the CUDA code uses for weights and gradients):
    W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3[1]   -> 5313 numbers
"""
from __future__ import annotations

import numpy as np

NIN, NH = 16, 64
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("w3", (NH,)), ("b3", (1,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest, ties to even) and back to float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def forward(params: dict, x: np.ndarray):
    """params: weights already in the precision the device uses (W* BF16-rounded, biases FP32)."""
    x = x.astype(np.float32)
    z1 = x @ params["W1"].T.astype(np.float32) + params["b1"]
    h1 = np.maximum(z1, 0).astype(np.float32)
    z2 = h1 @ params["W2"].T.astype(np.float32) + params["b2"]
    h2 = np.maximum(z2, 0).astype(np.float32)
    y = h2 @ params["w3"].astype(np.float32) + params["b3"][0]
    return y.astype(np.float32), (x, z1, h1, z2, h2)


def loss_and_grads(params: dict, x: np.ndarray, t: np.ndarray):
    """Mean squared error and its gradient with respect to every parameter (flat, float64)."""
    y, (x, z1, h1, z2, h2) = forward(params, x)
    n = x.shape[0]
    d = (y.astype(np.float64) - t.astype(np.float64))
    loss = float(np.mean(d * d))
    dy = 2.0 * d / n
    g = {}
    g["w3"] = h2.astype(np.float64).T @ dy
    g["b3"] = np.array([dy.sum()])
    dh2 = np.outer(dy, params["w3"].astype(np.float64)) * (z2 > 0)
    g["W2"] = dh2.T @ h1.astype(np.float64)
    g["b2"] = dh2.sum(axis=0)
    dh1 = (dh2 @ params["W2"].astype(np.float64)) * (z1 > 0)
    g["W1"] = dh1.T @ x.astype(np.float64)
    g["b1"] = dh1.sum(axis=0)
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])
    return loss, flat
