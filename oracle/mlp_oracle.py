"""TEST INFRASTRUCTURE ONLY -- CPU restatement (float64 numpy) of the
minimizer-order network, used to check the CUDA forward and backward kernels
(rapidgkc_b200/csrc/order_mlp.cu).  Nothing in the product imports it.

The reference has no learned order (its order is the fixed value order with
the "rapidgkc" filter, minimizer_filter.h:20, gpu_skmgen.cu:243-252); this is
the network that replaces that order:

  input   one-hot p-mer: 4p values, input 4*pos + base is 1 where `base` is the
          2-bit code (A=0 C=1 G=2 T=3) of position `pos`, pos 0 = first base
          (the most significant bits of the p-mer value)
  layer 1 h1 = relu(b1 + W1^T x)     W1: [4p][64]
  layer 2 h2 = relu(b2 + W2^T h1)    W2: [64][64]
  output  y  = b3 + w3 . h2          w3: [64]
  loss    L  = sum_s wt_s (y_s - t_s)^2 / sum_s wt_s

Parameters are one float32 vector, in this order: W1 (row-major [4p][64]),
b1, W2 (row-major [64][64], row = input unit), b2, w3, b3.
"""
from __future__ import annotations

import numpy as np

H = 64


def n_params(p: int) -> int:
    return 4 * p * H + H + H * H + H + H + 1


def unpack(params: np.ndarray, p: int):
    q = np.asarray(params, np.float64)
    o = 0
    W1 = q[o:o + 4 * p * H].reshape(4 * p, H); o += 4 * p * H
    b1 = q[o:o + H]; o += H
    W2 = q[o:o + H * H].reshape(H, H); o += H * H
    b2 = q[o:o + H]; o += H
    w3 = q[o:o + H]; o += H
    b3 = q[o]
    return W1, b1, W2, b2, w3, b3


def init_params(p: int, seed: int) -> np.ndarray:
    """He-normal weights, zero biases (float32)."""
    r = np.random.default_rng(seed)
    W1 = r.normal(0.0, np.sqrt(2.0 / p), (4 * p, H))  # p inputs are 1 per sample
    W2 = r.normal(0.0, np.sqrt(2.0 / H), (H, H))
    w3 = r.normal(0.0, np.sqrt(1.0 / H), H)
    return np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), w3, [0.0]]).astype(np.float32)


def one_hot(v: np.ndarray, p: int) -> np.ndarray:
    v = np.asarray(v, np.uint64)
    x = np.zeros((len(v), 4 * p))
    for pos in range(p):
        base = (v >> np.uint64(2 * (p - 1 - pos))) & np.uint64(3)
        x[np.arange(len(v)), 4 * pos + base.astype(np.int64)] = 1.0
    return x


def forward(params, p, v):
    W1, b1, W2, b2, w3, b3 = unpack(params, p)
    x = one_hot(v, p)
    h1 = np.maximum(x @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ w3 + b3


def loss_and_grad(params, p, v, t, wt=None):
    """Weighted mean squared error and its gradient (same layout as params)."""
    W1, b1, W2, b2, w3, b3 = unpack(params, p)
    t = np.asarray(t, np.float64)
    wt = np.ones_like(t) if wt is None else np.asarray(wt, np.float64)
    x = one_hot(v, p)
    a1 = x @ W1 + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ w3 + b3
    W = wt.sum()
    L = float((wt * (y - t) ** 2).sum() / W)
    dy = 2.0 * wt * (y - t) / W
    dw3 = h2.T @ dy
    db3 = dy.sum()
    dh2 = np.outer(dy, w3) * (a2 > 0)
    dW2 = h1.T @ dh2
    db2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (a1 > 0)
    dW1 = x.T @ dh1
    db1 = dh1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, [db3]])
    return L, g
