"""Test infrastructure (checker only): a NumPy restatement of the cost-model
network that libkifmm_b200's kfmm_mlp_* kernels implement, used to check
their forward pass and gradients.  Same packed parameter layout
[W1 | b1 | W2 | b2 | W3 | b3] (weights input-index major), same loss
mean((Y - T)^2).  Computes in float64 unless told otherwise.  The reference
has no such network, so this is pinned by a finite-difference check of its
own gradients (tests/test_costmodel.py) instead of reference vectors.
"""
import numpy as np


def unpack(p, F, H, O):
    sizes = [F * H, H, H * H, H, H * O, O]
    out, k = [], 0
    for s in sizes:
        out.append(p[k:k + s])
        k += s
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(F, H), b1, W2.reshape(H, H), b2, W3.reshape(H, O), b3


def forward(p, X, F, H, O, dtype=np.float64):
    W1, b1, W2, b2, W3, b3 = [a.astype(dtype) for a in unpack(np.asarray(p), F, H, O)]
    X = np.asarray(X, dtype)
    H1 = np.maximum(X @ W1 + b1, 0)
    H2 = np.maximum(H1 @ W2 + b2, 0)
    return H2 @ W3 + b3, (X, H1, H2)


def loss_and_gradients(p, X, T, F, H, O, dtype=np.float64):
    W1, b1, W2, b2, W3, b3 = [a.astype(dtype) for a in unpack(np.asarray(p), F, H, O)]
    Y, (X, H1, H2) = forward(p, X, F, H, O, dtype)
    T = np.asarray(T, dtype)
    n = Y.size
    loss = float(np.mean((Y - T) ** 2))
    dY = 2.0 * (Y - T) / n
    gW3, gb3 = H2.T @ dY, dY.sum(0)
    dH2 = (dY @ W3.T) * (H2 > 0)
    gW2, gb2 = H1.T @ dH2, dH2.sum(0)
    dH1 = (dH2 @ W2.T) * (H1 > 0)
    gW1, gb1 = X.T @ dH1, dH1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
