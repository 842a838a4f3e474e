"""CPU reference of the learned Newton start (TEST INFRASTRUCTURE ONLY).

numpy restatement of the net the library evaluates and trains on the GPU (the
kernels in enzo-dev_b200/csrc/ppm_guess.cuh and ppm_mlp.cu): a 6 -> 64 -> 64 -> 1
ReLU MLP with inputs, weights and hidden activations rounded to BF16 (round to
nearest even) and sums in higher precision.  It is the checker of the GPU gradients
and of the tensor-core inference, never part of the product path.

The net is not part of the reference code; the quantities it feeds are: the acoustic
start of twoshock.F:156-170 and the converged star pressure of twoshock.F:178-254.
"""
from __future__ import annotations

import numpy as np

NIN, NH = 6, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + NIN * NH
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NWEIGHTS = OFF_B3 + 1


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(w):
    w = np.asarray(w, dtype=np.float32)
    return (w[OFF_W1:OFF_B1].reshape(NIN, NH), w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH),
            w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3])


def init_weights(seed=0):
    """He-style initial weights (the training script's starting point)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NWEIGHTS, dtype=np.float32)
    w[OFF_W1:OFF_B1] = rng.standard_normal(NIN * NH) * np.sqrt(2.0 / NIN)
    w[OFF_W2:OFF_B2] = rng.standard_normal(NH * NH) * np.sqrt(2.0 / NH)
    w[OFF_W3:OFF_B3] = rng.standard_normal(NH) * np.sqrt(1.0 / NH)
    return w


def forward(w, x, rounding=True):
    """Net output for inputs x (n, 6); returns (y, cache) with float64 sums."""
    w = np.asarray(w)
    W1 = w[OFF_W1:OFF_B1].reshape(NIN, NH)
    b1, W2 = w[OFF_B1:OFF_W2], w[OFF_W2:OFF_B2].reshape(NH, NH)
    b2, w3, b3 = w[OFF_B2:OFF_W3], w[OFF_W3:OFF_B3], w[OFF_B3]
    if rounding:  # BF16 operands and activations, as the GPU computes them
        def r(a):
            return bf16(np.asarray(a, dtype=np.float32)).astype(np.float64)
    else:         # exact float64 (for finite-difference checks of the gradient)
        def r(a):
            return np.asarray(a, dtype=np.float64)
    xq = r(x)
    W1q, W2q, w3q = r(W1), r(W2), r(w3)
    z1 = xq @ W1q + np.asarray(b1, dtype=np.float64)
    h1 = r(np.maximum(z1, 0.0))
    z2 = h1 @ W2q + np.asarray(b2, dtype=np.float64)
    h2 = r(np.maximum(z2, 0.0))
    y = h2 @ w3q + float(b3)
    return y, (xq, z1, h1, z2, h2, W1q, W2q, w3q)


def loss_and_grad(w, samples, rounding=True):
    """Mean squared error over samples (n, 8: 6 inputs, target, weight) and its gradient
    with the rounding treated as the identity (as the GPU backward does)."""
    x = samples[:, :NIN]
    t = samples[:, 6].astype(np.float64)
    wt = samples[:, 7].astype(np.float64)
    n = samples.shape[0]
    y, (xq, z1, h1, z2, h2, W1q, W2q, w3q) = forward(w, x, rounding)
    err = y - t
    loss_sum = float(np.sum(wt * err * err))
    dy = wt * 2.0 * err / n
    g = np.zeros(NWEIGHTS, dtype=np.float64)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = (dy[:, None] * w3q[None, :]) * (z2 > 0)
    g[OFF_W2:OFF_B2] = (h1.T @ dz2).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    dz1 = (dz2 @ W2q.T) * (z1 > 0)
    g[OFF_W1:OFF_B1] = (xq.T @ dz1).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    return loss_sum, g


def features(dl, dr, pl, pr, ul, ur, gamma):
    """Inputs of the net and |x|^2 (float32, as the device computes them)."""
    rho = 0.5 * (dl + dr)
    p = 0.5 * (pl + pr)
    u = 0.5 * (ul + ur)
    c = np.sqrt(gamma * p / rho)
    f = np.stack([np.log(dl / rho), np.log(dr / rho), (ul - u) / c, (ur - u) / c,
                  np.log(pl / p), np.log(pr / p)], axis=-1).astype(np.float32)
    d2 = np.zeros(f.shape[:-1], dtype=np.float32)
    for k in range(6):
        d2 = (d2 + f[..., k] * f[..., k]).astype(np.float32)
    return f, d2


def acoustic_start(dl, dr, pl, pr, ul, ur, gamma, pmin):
    """twoshock.F:156-170."""
    cl = np.sqrt(gamma * pl * dl)
    cr = np.sqrt(gamma * pr * dr)
    ps = (cr * pl + cl * pr + cr * cl * (ul - ur)) / (cr + cl)
    return np.maximum(ps, pmin)


def samples_from_records(rec, gamma, pmin):
    """Log records (n, 8) -> training samples (n, 8), as ppm_b200_guess_features."""
    dl, dr, pl, pr, ul, ur, pstar, it = (rec[:, k] for k in range(8))
    f, d2 = features(dl, dr, pl, pr, ul, ur, gamma)
    ps = acoustic_start(dl, dr, pl, pr, ul, ur, gamma, pmin)
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.log(pstar / ps) / d2.astype(np.float64)
    ok = (it > 0) & (d2 > 1e-12) & np.isfinite(t) & (np.abs(t) < 16.0)
    ok &= np.all(np.isfinite(f), axis=1)
    out = np.zeros((rec.shape[0], 8), dtype=np.float32)
    out[:, :6] = f
    out[:, 6] = np.where(ok, t, 0.0)
    out[:, 7] = ok.astype(np.float32)
    return out
