"""CPU restatement of the threshold predictor's network, for checking the CUDA kernels (mlp.cu).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU forward pass and gradients;
nothing in the product calls it. Float64 throughout.

Network: y = w3 . gelu(W2^T gelu(W1^T x + b1) + b2) + b3 with the exact (erf) GELU, parameters in one
flat vector W1 [din][H], b1 [H], W2 [H][H], b2 [H], w3 [H], b3 [1]; loss = mean((y - t)^2), or with
tau in (0, 1) the pinball loss of the tau-quantile, mean(tau (t - y) where t >= y, (1 - tau) (y - t)
elsewhere).
"""
import math

import numpy as np

_erf = np.vectorize(math.erf)


def unpack(p, din, h):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + din * h].reshape(din, h)
    o += din * h
    b1 = p[o:o + h]
    o += h
    W2 = p[o:o + h * h].reshape(h, h)
    o += h * h
    b2 = p[o:o + h]
    o += h
    w3 = p[o:o + h]
    o += h
    return W1, b1, W2, b2, w3, p[o]


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(p, X, din, h):
    W1, b1, W2, b2, w3, b3 = unpack(p, din, h)
    X = np.asarray(X, np.float64)
    Z1 = X @ W1 + b1
    A1 = gelu(Z1)
    Z2 = A1 @ W2 + b2
    A2 = gelu(Z2)
    return A2 @ w3 + b3, (X, Z1, A1, Z2, A2)


def loss_and_grad(p, X, t, din, h, tau=0.0):
    """(loss, its gradient as a flat vector in parameter order): the mean squared error for tau = 0,
    else the pinball loss of the tau-quantile."""
    W1, b1, W2, b2, w3, b3 = unpack(p, din, h)
    y, (X, Z1, A1, Z2, A2) = forward(p, X, din, h)
    t = np.asarray(t, np.float64)
    d = y - t
    if tau <= 0.0:
        loss = float(np.mean(d * d))
        dy = 2.0 * d / len(t)
    else:
        loss = float(np.mean(np.where(d > 0, (1.0 - tau) * d, -tau * d)))
        dy = np.where(d > 0, 1.0 - tau, -tau) / len(t)
    gw3 = A2.T @ dy
    gb3 = dy.sum()
    dZ2 = np.outer(dy, w3) * gelu_grad(Z2)
    gW2 = A1.T @ dZ2
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * gelu_grad(Z1)
    gW1 = X.T @ dZ1
    gb1 = dZ1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
