"""ORACLE (test infrastructure only): numpy restatement of the learned-settings
MLP -- forward pass, mean-squared-error gradient and Adam step -- in float64.

It restates the arithmetic of jxpamg_all_b200/csrc/learned.cu (the network
has no counterpart in the reference): x_n = (x - mu) / sigma,
h = tanh(W1 x_n + b1), y = W2 h + b2, loss = mean over samples and outputs of
(y - t)^2; mu and sigma are fixed (zero gradient); Adam with bias correction
updates every other weight.  Tests compare the CUDA kernels against these
functions and check these against finite differences.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HIDDEN, N_OUT = 16, 64, 3
OFF_MU, OFF_SIGMA, OFF_W1 = 0, 16, 32
OFF_B1 = OFF_W1 + N_HIDDEN * N_IN
OFF_W2 = OFF_B1 + N_HIDDEN
OFF_B2 = OFF_W2 + N_OUT * N_HIDDEN
N_WEIGHTS = OFF_B2 + N_OUT


def _split(w):
    w = np.asarray(w, np.float64)
    return (w[OFF_MU:OFF_SIGMA], w[OFF_SIGMA:OFF_W1], w[OFF_W1:OFF_B1].reshape(N_HIDDEN, N_IN), w[OFF_B1:OFF_W2],
            w[OFF_W2:OFF_B2].reshape(N_OUT, N_HIDDEN), w[OFF_B2:])


def forward(w, X):
    """Returns (Y [B,3], H [B,64], Xn [B,16])."""
    mu, sg, W1, b1, W2, b2 = _split(w)
    Xn = (np.asarray(X, np.float64) - mu) / sg
    H = np.tanh(Xn @ W1.T + b1)
    return H @ W2.T + b2, H, Xn


def loss_grad(w, X, T):
    """Mean squared error over samples and outputs and its gradient (N_WEIGHTS)."""
    Y, H, Xn = forward(w, X)
    B = Y.shape[0]
    _, _, W1, _, W2, _ = _split(w)
    D = Y - np.asarray(T, np.float64)
    loss = float(np.mean(D * D))
    dY = 2.0 * D / (N_OUT * B)
    dZ = (dY @ W2) * (1.0 - H * H)
    g = np.zeros(N_WEIGHTS)
    g[OFF_W1:OFF_B1] = (dZ.T @ Xn).reshape(-1)
    g[OFF_B1:OFF_W2] = dZ.sum(axis=0)
    g[OFF_W2:OFF_B2] = (dY.T @ H).reshape(-1)
    g[OFF_B2:] = dY.sum(axis=0)
    return loss, g


def adam_step(w, g, m, v, lr, beta1, beta2, eps, step):
    """One Adam update of every weight after mu and sigma; returns (w, m, v)."""
    w, m, v = (np.array(a, np.float64) for a in (w, m, v))
    c1, c2 = 1.0 - beta1 ** step, 1.0 - beta2 ** step
    sl = slice(OFF_W1, N_WEIGHTS)
    m[sl] = beta1 * m[sl] + (1 - beta1) * g[sl]
    v[sl] = beta2 * v[sl] + (1 - beta2) * g[sl] * g[sl]
    w[sl] -= lr * (m[sl] / c1) / (np.sqrt(v[sl] / c2) + eps)
    return w, m, v
