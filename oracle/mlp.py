"""CPU oracle of the surrogate MLP: forward pass, backward pass and Adam step in
numpy.  Test infrastructure only: the library's surrogate runs on the tensor
cores (dem_mlp_* kernels); this file is what its outputs and gradients are
checked against.

The reference's surrogate is sklearn's MLPRegressor (NN_MP.py:374-378, fitted
at NN_MP.py:895, evaluated at NN_MP.py:384-395): dense layers
a_{l} = act(a_{l-1} W_l^T + b_l) with ReLU hidden units and an identity output,
squared-error loss, Adam (beta1 0.9, beta2 0.999, eps 1e-8) and an L2 penalty.
It is a third-party dependency (scikit-learn, not vendored in the reference;
this image carries 1.9.0), so parity is anchored on calling it: the float64
path of this file (bf16=False) reproduces MLPRegressor's predictions and its
backprop gradients (tests/test_mlp_oracle.py).  The bf16=True path restates
what the device computes: every GEMM operand (inputs, weights, hidden
activations, output and hidden-layer gradients) rounded to bfloat16 (round to
nearest even), products accumulated in float32 or better, pre-activations,
gradients and master weights in float32.  GELU is the tanh form (the device
evaluates its tanh with the hardware approximation, relative error about
2^-11; this file with numpy's tanh).

Weights follow the device layout: W_l has shape (out, in) (sklearn's coefs_
are the transposes), loss = mean over all rows and outputs of (y - t)^2.
"""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


GELU_C, GELU_A = np.sqrt(2.0 / np.pi), 0.044715


def act(z: np.ndarray, kind: str) -> np.ndarray:
    """ReLU, or GELU in the tanh form of Hendrycks & Gimpel (2016):
    z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    if kind == "relu":
        return np.maximum(z, 0)
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def act_grad(z: np.ndarray, kind: str) -> np.ndarray:
    """Derivative of act (ReLU: 0 at 0, as sklearn)."""
    if kind == "relu":
        return (z > 0).astype(z.dtype)
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def _mm(a, b, rnd):
    """a @ b with bf16 operands (rnd) accumulated in float64, or plain float64."""
    if rnd:
        return (bf16(a).astype(np.float64) @ bf16(b).astype(np.float64)).astype(np.float32)
    return a.astype(np.float64) @ b.astype(np.float64)


def forward(W: list, b: list, x: np.ndarray, kind: str = "gelu", rnd: bool = True):
    """Returns (y, zs, hs): output, pre-activations of the hidden layers, and the
    layer inputs hs[0] = x, hs[l] = act(zs[l-1]) (bf16-rounded when rnd)."""
    h = bf16(x) if rnd else x.astype(np.float64)
    hs, zs = [h], []
    for l, (Wl, bl) in enumerate(zip(W, b)):
        z = _mm(h, Wl.T, rnd) + (bl.astype(np.float32) if rnd else bl.astype(np.float64))
        if l == len(W) - 1:
            return z, zs, hs
        zs.append(z)
        h = act(z, kind)
        h = bf16(h) if rnd else h
        hs.append(h)
    raise ValueError("no layers")


def backward(W: list, b: list, x: np.ndarray, t: np.ndarray, kind: str = "gelu", rnd: bool = True,
             input_grad: bool = False):
    """Gradients of mean((y - t)^2) with respect to W, b (and x).  Returns
    (loss, dW, db, dx)."""
    y, zs, hs = forward(W, b, x, kind, rnd)
    n = y.size
    d = 2.0 * (y - t) / n
    d = d.astype(np.float32) if rnd else d
    loss = float(np.mean((y.astype(np.float64) - t) ** 2))
    dW, db = [None] * len(W), [None] * len(W)
    dx = None
    for l in range(len(W) - 1, -1, -1):
        dW[l] = _mm(d.T, hs[l], rnd)
        db[l] = d.sum(axis=0, dtype=np.float64).astype(d.dtype)
        if l == 0 and not input_grad:
            break
        dh = _mm(d, W[l], rnd)
        if l == 0:
            dx = dh
            break
        d = dh * act_grad(zs[l - 1], kind)
        d = d.astype(np.float32) if rnd else d
    return loss, dW, db, dx


def adam(w, g, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, l2=0.0):
    """One Adam step (bias-corrected, gradient g + l2 w); returns new (w, m, v)."""
    g = g + l2 * w
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** t)) / (np.sqrt(v / (1 - b2 ** t)) + eps)
    return w, m, v
