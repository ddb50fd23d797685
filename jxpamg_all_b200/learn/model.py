"""Weight layout and output maps of the learned-settings MLP (host side).

The layout matches jxpamg_all_b200/csrc/learned.cuh: one float32 blob
mu[16], sigma[16], W1[64][16], b1[64], W2[3][64], b2[3].  Outputs are logits:
theta = 0.1 + 0.8 s(y0), lower = 0.02 + 0.68 s(y1), upper = 0.8 + 0.7 s(y2)
with s the logistic function; the Chebyshev interval is [lower, upper] x
lambda_max(D^-1 A).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HIDDEN, N_OUT = 16, 64, 3
OFF_MU, OFF_SIGMA = 0, 16
OFF_W1 = 32
OFF_B1 = OFF_W1 + N_HIDDEN * N_IN
OFF_W2 = OFF_B1 + N_HIDDEN
OFF_B2 = OFF_W2 + N_OUT * N_HIDDEN
N_WEIGHTS = OFF_B2 + N_OUT


def _sig(y):
    return 1.0 / (1.0 + np.exp(-np.asarray(y, dtype=np.float64)))


def theta_of(y):
    return 0.1 + 0.8 * _sig(y)


def lower_of(y):
    return 0.02 + 0.68 * _sig(y)


def upper_of(y):
    return 0.8 + 0.7 * _sig(y)


def _logit(p):
    p = np.clip(np.asarray(p, dtype=np.float64), 1e-4, 1 - 1e-4)
    return np.log(p / (1 - p))


def to_logits(theta, lower, upper):
    """Inverse of the output maps: settings -> target logits [..., 3]."""
    return np.stack([_logit((np.asarray(theta) - 0.1) / 0.8), _logit((np.asarray(lower) - 0.02) / 0.68),
                     _logit((np.asarray(upper) - 0.8) / 0.7)], axis=-1)


def pack(mu, sigma, W1, b1, W2, b2):
    w = np.zeros(N_WEIGHTS, np.float32)
    w[OFF_MU:OFF_MU + N_IN] = mu
    w[OFF_SIGMA:OFF_SIGMA + N_IN] = sigma
    w[OFF_W1:OFF_B1] = np.asarray(W1, np.float32).reshape(-1)
    w[OFF_B1:OFF_W2] = b1
    w[OFF_W2:OFF_B2] = np.asarray(W2, np.float32).reshape(-1)
    w[OFF_B2:] = b2
    return w


def unpack(w):
    w = np.asarray(w, np.float32)
    return dict(mu=w[OFF_MU:OFF_MU + N_IN], sigma=w[OFF_SIGMA:OFF_SIGMA + N_IN],
                W1=w[OFF_W1:OFF_B1].reshape(N_HIDDEN, N_IN), b1=w[OFF_B1:OFF_W2],
                W2=w[OFF_W2:OFF_B2].reshape(N_OUT, N_HIDDEN), b2=w[OFF_B2:])


def init_weights(rng, mu, sigma):
    W1 = rng.standard_normal((N_HIDDEN, N_IN)) * np.sqrt(1.0 / N_IN)
    W2 = rng.standard_normal((N_OUT, N_HIDDEN)) * np.sqrt(1.0 / N_HIDDEN) * 0.1
    return pack(mu, sigma, W1, np.zeros(N_HIDDEN), W2, np.zeros(N_OUT))


def write_weights_inc(path, w, note):
    """C initialiser compiled into the library (csrc/learned_weights.inc)."""
    w = np.asarray(w, np.float32)
    assert w.shape == (N_WEIGHTS,)
    rows = [", ".join(f"{float(v):.8e}f" for v in w[i:i + 6]) for i in range(0, N_WEIGHTS, 6)]
    with open(path, "w") as f:
        f.write("// MLP weights compiled into the library (layout: mu[16], sigma[16], W1[64][16], b1[64], "
                "W2[3][64], b2[3]).\n")
        f.write(f"// {note}\n")
        f.write(f"const float kDefaultMlpWeights[{N_WEIGHTS}] = {{\n")
        f.write(",\n".join(rows))
        f.write("\n};\n")
