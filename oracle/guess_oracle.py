"""CPU restatement of the learned recovery guess's network, for the tests only
(TEST INFRASTRUCTURE: nothing in the product imports this file).

The device computes an MLP 8 -> 64 -> 64 -> 3 with GELU on the tensor cores:
operands rounded to BF16, products accumulated in FP32, biases and activations
in FP32 (fivohydro.jl_b200/csrc/guess.cuh). `forward`/`grad` below round at the
same places (`bf16`), so they agree with the device to FP32 accumulation order;
`forward64`/`grad64` are the same network in plain float64 (no rounding), which
the tests check against finite differences to pin the backward pass itself.

Parameter vector (FIVO_GUESS_NPARAM floats): W1[64][16] b1[64] W2[64][64]
b2[64] W3[16][64] b3[16], W[out][in]; W1's columns 8..15, W3's rows 3..15 and
b3[3..15] are padding. Samples: 8 raw features, 3 raw targets. The reference
has no counterpart (its Newton starts from the previous step or a closed-form
seed, src2d/primrec2d.jl:300-347,465-486).
"""
from __future__ import annotations

import math

import numpy as np

NIN, K0, NH, NOUT, N3 = 8, 16, 64, 3, 16
P_W1 = 0
P_B1 = P_W1 + NH * K0
P_W2 = P_B1 + NH
P_B2 = P_W2 + NH * NH
P_W3 = P_B2 + NH
P_B3 = P_W3 + N3 * NH
NPARAM = P_B3 + N3

_erf = np.vectorize(math.erf)


def bf16(x):
    """round to bfloat16 (nearest even) and back to float32"""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    W1 = P[P_W1:P_B1].reshape(NH, K0)
    b1 = P[P_B1:P_W2]
    W2 = P[P_W2:P_B2].reshape(NH, NH)
    b2 = P[P_B2:P_W3]
    W3 = P[P_W3:P_B3].reshape(N3, NH)
    b3 = P[P_B3:NPARAM]
    return W1, b1, W2, b2, W3, b3


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def normalise(norm, raw):
    """x_n = clamp((r - mean) * istd, -8, 8) in float32 (norm: 22 floats)"""
    norm = np.asarray(norm, dtype=np.float32)
    r = np.asarray(raw, dtype=np.float32)[:, :NIN]
    x = (r - norm[:8]) * norm[8:16]
    return np.clip(x, -8.0, 8.0).astype(np.float32)


def norm_targets(norm, samples):
    norm = np.asarray(norm, dtype=np.float32)
    t = np.asarray(samples, dtype=np.float32)[:, NIN:NIN + NOUT]
    return ((t - norm[16:19]) / norm[19:22]).astype(np.float32)


def _mm(a, b):
    """a @ b of BF16-valued float32 operands, accumulated exactly and rounded to float32"""
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)


def forward(P, xn):
    """device-rounded forward: normalised outputs (n, 3) and the cache for grad"""
    W1, b1, W2, b2, W3, b3 = (np.asarray(w, dtype=np.float32) for w in unpack(P))
    X = np.zeros((xn.shape[0], K0), dtype=np.float32)
    X[:, :NIN] = xn
    Xb = bf16(X)
    z1 = (_mm(Xb, bf16(W1).T) + b1).astype(np.float32)
    h1 = bf16(gelu(z1.astype(np.float64)).astype(np.float32))
    z2 = (_mm(h1, bf16(W2).T) + b2).astype(np.float32)
    h2 = bf16(gelu(z2.astype(np.float64)).astype(np.float32))
    y = (_mm(h2, bf16(W3).T) + b3).astype(np.float32)
    return y[:, :NOUT], (Xb, z1, h1, z2, h2, y)


def grad(P, norm, samples):
    """device-rounded gradient of the mean over samples of sum_o (y_o - t_o)^2,
    and that loss"""
    xn = normalise(norm, samples)
    tn = norm_targets(norm, samples)
    n = xn.shape[0]
    W1, b1, W2, b2, W3, b3 = (np.asarray(w, dtype=np.float32) for w in unpack(P))
    _, (Xb, z1, h1, z2, h2, y) = forward(P, xn)
    e = y[:, :NOUT] - tn
    loss = float(np.sum(e.astype(np.float64) ** 2) / n)
    dy = np.zeros((n, N3), dtype=np.float32)
    dy[:, :NOUT] = 2.0 * e * np.float32(1.0 / n)
    dyb = bf16(dy)
    dh2 = _mm(dyb, bf16(W3))                         # (n, 64)
    dz2 = (dh2 * gelu_d(z2.astype(np.float64)).astype(np.float32)).astype(np.float32)
    dz2b = bf16(dz2)
    dh1 = _mm(dz2b, bf16(W2))
    dz1 = (dh1 * gelu_d(z1.astype(np.float64)).astype(np.float32)).astype(np.float32)
    dz1b = bf16(dz1)
    G = np.zeros(NPARAM, dtype=np.float64)
    G[P_W1:P_B1] = _mm(dz1b.T, Xb).ravel()
    G[P_B1:P_W2] = dz1.astype(np.float64).sum(0)
    G[P_W2:P_B2] = _mm(dz2b.T, h1).ravel()
    G[P_B2:P_W3] = dz2.astype(np.float64).sum(0)
    G[P_W3:P_B3] = _mm(dyb.T, h2).ravel()
    G[P_B3:P_B3 + NOUT] = dy[:, :NOUT].astype(np.float64).sum(0)
    return G, loss


def loss64(P, xn, tn):
    """the loss of the float64 network without any rounding"""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    X = np.zeros((xn.shape[0], K0))
    X[:, :NIN] = xn
    h1 = gelu(X @ W1.T + b1)
    h2 = gelu(h1 @ W2.T + b2)
    y = (h2 @ W3.T + b3)[:, :NOUT]
    return float(np.sum((y - tn) ** 2) / xn.shape[0])


def grad64(P, xn, tn):
    """backpropagation of loss64 (float64, no rounding)"""
    W1, b1, W2, b2, W3, b3 = unpack(P)
    n = xn.shape[0]
    X = np.zeros((n, K0))
    X[:, :NIN] = xn
    z1 = X @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    y = h2 @ W3.T + b3
    dy = np.zeros((n, N3))
    dy[:, :NOUT] = 2.0 * (y[:, :NOUT] - tn) / n
    dz2 = (dy @ W3) * gelu_d(z2)
    dz1 = (dz2 @ W2) * gelu_d(z1)
    G = np.zeros(NPARAM)
    G[P_W1:P_B1] = (dz1.T @ X).ravel()
    G[P_B1:P_W2] = dz1.sum(0)
    G[P_W2:P_B2] = (dz2.T @ h1).ravel()
    G[P_B2:P_W3] = dz2.sum(0)
    G[P_W3:P_B3] = (dy.T @ h2).ravel()
    G[P_B3:NPARAM] = dy.sum(0)
    return G
