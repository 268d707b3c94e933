"""FP64 numpy restatement of the condensation surrogate (test infrastructure: the CPU checker of
the GPU forward, backward and inference kernels of cleo_b200/csrc/mlp.cu).

Parameter vector: W1[64][7], b1[64], W2[64][64], b2[64], W3[64], b3 (4737 floats). Normalisation
vector: feature means[7], feature inverse scales[7], target mean, target scale.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import erf

NIN, NH = 7, 64
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3 = 0, 448, 512, 4608, 4672, 4736
NPARAM = 4737
GROUPS = {"W1": (OFF_W1, OFF_B1), "b1": (OFF_B1, OFF_W2), "W2": (OFF_W2, OFF_B2),
          "b2": (OFF_B2, OFF_W3), "W3": (OFF_W3, OFF_B3), "b3": (OFF_B3, NPARAM)}


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(NH, NIN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NH, NH),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)


def standardise(feats, target, norm):
    norm = np.asarray(norm, dtype=np.float64)
    x = (np.asarray(feats, dtype=np.float64) - norm[:NIN]) * norm[NIN:2 * NIN]
    t = None if target is None else (np.asarray(target, dtype=np.float64) - norm[14]) / norm[15]
    return x, t


def loss_grad(p, norm, feats, target):
    """Mean squared error of the standardised target and its gradient (FP64)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x, t = standardise(feats, target, norm)
    a1 = x @ W1.T + b1
    h1 = gelu(a1)
    a2 = h1 @ W2.T + b2
    h2 = gelu(a2)
    y = h2 @ W3 + b3
    d = y - t
    n = len(t)
    loss = float((d * d).sum() / n)
    dy = 2.0 * d / n
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    da2 = dy[:, None] * W3[None, :] * gelu_grad(a2)
    g[OFF_W2:OFF_B2] = (da2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = da2.sum(0)
    da1 = (da2 @ W2) * gelu_grad(a1)
    g[OFF_W1:OFF_B1] = (da1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = da1.sum(0)
    return loss, g


def bf16_round(a):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def infer_bf16(p, norm, feats):
    """The inference function of the GPU kernels: BF16-rounded W1, W2, W3 and hidden layer 1,
    evaluated in FP64. Returns the denormalised prediction."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    x, _ = standardise(np.asarray(feats, dtype=np.float32), None, np.asarray(norm, np.float32))
    h1 = bf16_round(gelu(x @ W1.T + b1))
    y = gelu(h1 @ W2.T + b2) @ W3 + b3
    norm = np.asarray(norm, dtype=np.float64)
    return norm[14] + norm[15] * y
