"""CPU ORACLE of the learned strip's MLP — TEST INFRASTRUCTURE ONLY.

A plain numpy restatement, in FP64, of the network that
staggered-grid_b200/csrc/learned.cu evaluates and trains on the GPU: 252
inputs, two hidden layers of 64 GELU units, 9 outputs; parameters flattened
as W1[252][64], b1[64], W2[64][64], b2[64], W3[64][9], b3[9]; loss the mean
of the squared errors over all rows and the 9 outputs.  Only tests/ use it,
to check the GPU's forward pass and gradients.  The reference has no such
network; the restatement follows the definition written in learned.cu.

`forward_f16` is the same network with the operand rounding of the GPU's
tensor-core inference (k_strip_tc): inputs, weights and both hidden
activations rounded to IEEE binary16 (round to nearest even), biases and all
sums exact (FP64 here, FP32 accumulators on the GPU).
"""
import math

import numpy as np

N_IN, N_H, N_OUT = 252, 64, 9
SHAPES = [("W1", (N_IN, N_H)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)), ("W3", (N_H, N_OUT)),
          ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    p = np.asarray(p, np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


_erf = np.vectorize(math.erf)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward(p, X):
    w = unpack(p)
    X = np.asarray(X, np.float64)
    z1 = X @ w["W1"] + w["b1"]
    a1 = gelu(z1)
    z2 = a1 @ w["W2"] + w["b2"]
    a2 = gelu(z2)
    return a2 @ w["W3"] + w["b3"], (X, z1, a1, z2, a2)


def f16(a):
    """Round to IEEE binary16 (nearest even) and back."""
    return np.asarray(a, np.float64).astype(np.float16).astype(np.float64)


def forward_f16(p, X):
    w = unpack(p)
    a1 = f16(gelu(f16(X) @ f16(w["W1"]) + w["b1"]))
    a2 = f16(gelu(a1 @ f16(w["W2"]) + w["b2"]))
    return a2 @ f16(w["W3"]) + w["b3"]


def loss_and_gradient(p, X, Y):
    w = unpack(p)
    out, (X, z1, a1, z2, a2) = forward(p, X)
    Y = np.asarray(Y, np.float64)
    n = out.size
    d = out - Y
    loss = float(np.sum(d * d) / n)
    d3 = 2.0 * d / n
    g = {"W3": a2.T @ d3, "b3": d3.sum(0)}
    d2 = (d3 @ w["W3"].T) * gelu_grad(z2)
    g["W2"], g["b2"] = a1.T @ d2, d2.sum(0)
    d1 = (d2 @ w["W2"].T) * gelu_grad(z1)
    g["W1"], g["b1"] = X.T @ d1, d1.sum(0)
    return loss, np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])
