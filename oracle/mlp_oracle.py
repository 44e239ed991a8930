"""Oracle for the learned plan selector's network: TEST INFRASTRUCTURE ONLY.

A float64 numpy restatement of the MLP F -> 64 -> 64 -> 1 (ReLU) that the GPU
library trains with its own CUDA kernels (forward, mean-squared-error
gradients, Adam). Tests compare the GPU gradients with these. The network has
no counterpart in the reference library (its autotuner is a stub,
selector/selector.c:989-1004); the parameter layout is the GPU library's:
W1[F][64], b1[64], W2[64][64], b2[64], w3[64], b3[1].
"""
import numpy as np

H = 64


def nparams(F):
    return F * H + H + H * H + H + H + 1


def unpack(p, F):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + F * H].reshape(F, H); o += F * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, F, X):
    W1, b1, W2, b2, w3, b3 = unpack(p, F)
    H1 = np.maximum(X @ W1 + b1, 0.0)
    H2 = np.maximum(H1 @ W2 + b2, 0.0)
    return H2 @ w3 + b3, H1, H2


def grad(p, F, X, t):
    """Gradient of mean((y - t)^2) with respect to the flat parameters, and the loss."""
    X = np.asarray(X, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p, F)
    y, H1, H2 = forward(p, F, X)
    B = X.shape[0]
    dy = 2.0 * (y - t) / B
    gw3 = H2.T @ dy
    gb3 = dy.sum()
    D2 = np.outer(dy, w3) * (H2 > 0)
    gW2 = H1.T @ D2
    gb2 = D2.sum(0)
    D1 = (D2 @ W2.T) * (H1 > 0)
    gW1 = X.T @ D1
    gb1 = D1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return g, float(np.mean((y - t) ** 2))
