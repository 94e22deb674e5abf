"""CPU oracle of the closure MLP (test infrastructure, never shipped).

The MLP 24 -> 64 -> 64 -> 2 with GELU, restated in numpy FP64. There is no closure in
the reference, so this oracle is the project's own definition of the network; its
gradients are pinned by finite differences (tests/test_closure_oracle.py).

`forward`/`gradients` with rounding=True apply BF16 rounding at the points where the
tensor-core kernels hold BF16 values (inputs, weights, H1, H2, dH2, dH1); rounding=False
is the exact FP64 network used for the finite-difference check.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

NIN, NH, NOUT = 24, 64, 2
SHAPES = (("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NOUT, NH)), ("b3", (NOUT,)))
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    bits = f.view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return bits.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def pack(p):
    return np.concatenate([np.asarray(p[name], dtype=np.float64).ravel() for name, _ in SHAPES])


# GELU in the tanh form of Hendrycks and Gimpel (2016), the network's activation:
# gelu(x) = x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))). It differs from the erf form
# x/2 (1 + erf(x / sqrt 2)) by at most 4.8e-4 (test_closure.py checks the bound).
GELU_C0 = np.sqrt(2.0 / np.pi)
GELU_C1 = 0.044715 * GELU_C0


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(x * (GELU_C0 + GELU_C1 * x * x)))


def gelu_grad(x):
    t = np.tanh(x * (GELU_C0 + GELU_C1 * x * x))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * (GELU_C0 + 3 * GELU_C1 * x * x)


def gelu_erf(x):
    """The erf form of GELU (Hendrycks and Gimpel 2016), for the bound above."""
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def forward(flat, X, rounding=True):
    p = unpack(flat)
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    X = r(X)
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    Z1 = X @ W1.T + p["b1"]
    H1 = r(gelu(Z1))
    Z2 = H1 @ W2.T + p["b2"]
    H2 = r(gelu(Z2))
    Y = H2 @ W3.T + p["b3"]
    return Y, (X, Z1, H1, Z2, H2, W1, W2, W3)


def loss(flat, X, T, rounding=True):
    Y, _ = forward(flat, X, rounding)
    return float(((Y - T) ** 2).sum() / len(X))


def gradients(flat, X, T, rounding=True):
    """Gradient of (1/n) sum_rows sum_k (y_k - t_k)^2, packed like the parameters."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    Y, (X, Z1, H1, Z2, H2, W1, W2, W3) = forward(flat, X, rounding)
    n = len(X)
    dY = 2.0 * (Y - T) / n
    g = {"W3": dY.T @ H2, "b3": dY.sum(axis=0)}
    dH2 = r((dY @ W3) * gelu_grad(Z2))
    g["W2"], g["b2"] = dH2.T @ H1, dH2.sum(axis=0)
    dH1 = r((dH2 @ W2) * gelu_grad(Z1))
    g["W1"], g["b1"] = dH1.T @ X, dH1.sum(axis=0)
    return pack(g), float(((Y - T) ** 2).sum() / n)


def init_params(seed: int = 0):
    """Seeded He-style initialization."""
    rng = np.random.default_rng(seed)
    p = {"W1": rng.standard_normal((NH, NIN)) * np.sqrt(2.0 / NIN), "b1": np.zeros(NH),
         "W2": rng.standard_normal((NH, NH)) * np.sqrt(2.0 / NH), "b2": np.zeros(NH),
         "W3": rng.standard_normal((NOUT, NH)) * np.sqrt(1.0 / NH), "b3": np.zeros(NOUT)}
    return pack(p)
