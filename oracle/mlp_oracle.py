"""CPU oracle of the warm-start MLP (test infrastructure only).

FP64 numpy forward and backward of the n_in -> H -> H -> n_out GELU network
with mean-squared-error loss, in the parameter layout of
ufem_mlp_get_params (W1 [H][32] with the inputs zero-padded to 32, b1,
W2 [H][H], b2, W3 [n_out][H], b3).  ``bf16=True`` rounds to BF16 exactly
where the GPU path feeds its tensor-core products (inputs, weights, hidden
activations, back-propagated gradients), so the two can be compared
closely; ``bf16=False`` is the plain FP64 reference used for the
finite-difference check of the analytic gradients.
"""
from __future__ import annotations

import math

import numpy as np

N_INP = 32


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even) and return as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split(params: np.ndarray, H: int, n_out: int):
    p = np.asarray(params, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * N_INP].reshape(H, N_INP); o += H * N_INP
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + n_out * H].reshape(n_out, H); o += n_out * H
    b3 = p[o:o + n_out]; o += n_out
    return W1, b1, W2, b2, W3, b3


def gelu(x):
    return 0.5 * x * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0)))
    return cdf + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward(params, X, H, n_out, bf=True):
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = split(params, H, n_out)
    Xp = np.zeros((X.shape[0], N_INP))
    Xp[:, :X.shape[1]] = X
    Xb = r(Xp)
    Z1 = Xb @ r(W1).T + b1
    H1 = r(gelu(Z1))
    Z2 = H1 @ r(W2).T + b2
    H2 = r(gelu(Z2))
    Y = H2 @ r(W3).T + b3
    return dict(Xb=Xb, Z1=Z1, H1=H1, Z2=Z2, H2=H2, Y=Y)


def loss_and_grads(params, X, T, H, n_out, bf=True):
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = split(params, H, n_out)
    f = forward(params, X, H, n_out, bf)
    B = X.shape[0]
    D = f["Y"] - T
    loss = float((D * D).sum() / (B * n_out))
    dY = 2.0 * D / (B * n_out)
    dYb = r(dY)
    gW3 = dYb.T @ f["H2"]
    gb3 = dY.sum(0)
    dZ2 = (dYb @ r(W3)) * gelu_grad(f["Z2"])
    dZ2b = r(dZ2)
    gW2 = dZ2b.T @ f["H1"]
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2b @ r(W2)) * gelu_grad(f["Z1"])
    dZ1b = r(dZ1)
    gW1 = dZ1b.T @ f["Xb"]
    gb1 = dZ1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
