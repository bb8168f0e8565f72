"""CPU reference of the surrogate network's forward pass and gradient.

TEST INFRASTRUCTURE ONLY: the checker for the rcwa_mlp_* kernels (``tests/``).
The network and its parameter layout follow include/rcwa_b200.h: layers of
W (out x in, row-major) then b (out); GELU (the exact, erf-based form) on
every hidden layer; loss = mean over all outputs of the squared error.
Computed in float64.
"""
from __future__ import annotations

import math

import numpy as np


def _erf(x):
    return np.vectorize(math.erf)(x)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def unpack(params, dims):
    out, o = [], 0
    for i in range(len(dims) - 1):
        n_in, n_out = dims[i], dims[i + 1]
        W = params[o:o + n_out * n_in].reshape(n_out, n_in)
        o += n_out * n_in
        b = params[o:o + n_out]
        o += n_out
        out.append((W.astype(np.float64), b.astype(np.float64)))
    return out


def forward(params, dims, X):
    layers = unpack(params, dims)
    H = [np.asarray(X, dtype=np.float64)]
    Z = []
    for i, (W, b) in enumerate(layers):
        z = H[-1] @ W.T + b
        Z.append(z)
        if i + 1 < len(layers):
            H.append(gelu(z))
    return Z[-1], H, Z


def loss_grad(params, dims, X, Y):
    layers = unpack(params, dims)
    P, H, Z = forward(params, dims, X)
    D = P - np.asarray(Y, dtype=np.float64)
    loss = float(np.mean(D * D))
    dz = 2.0 * D / D.size
    grads = [None] * len(layers)
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        grads[i] = (dz.T @ H[i], dz.sum(axis=0))
        if i > 0:
            dz = (dz @ W) * gelu_grad(Z[i - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
