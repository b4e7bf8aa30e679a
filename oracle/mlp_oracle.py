"""CPU oracle for the emulator network (test infrastructure only).

FP64 numpy restatement of the forward pass, the MSE loss and the backward
pass of the 5 -> 256 -> 256 -> 256 -> 1 SiLU network whose training kernels
live in ``cosmoforge_b200/csrc/mlp.cu``.  The emulator has no counterpart in
the reference, so this restatement is the checker of the device gradients:
it takes the same BF16-rounded weight matrices the device forward and
backward passes read (biases stay FP32 on the device and FP64 here), so
the comparison isolates the device's FP32 accumulation.  Only the tests
import this module.
"""

from __future__ import annotations

import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(flat, sizes):
    """Split the flat parameter vector into [(W, b), ...] with W of shape (out, in)."""
    out, off = [], 0
    for n_in, n_out in zip(sizes[:-1], sizes[1:]):
        W = flat[off: off + n_out * n_in].reshape(n_out, n_in)
        off += n_out * n_in
        b = flat[off: off + n_out]
        off += n_out
        out.append((W, b))
    return out


def forward(layers, X):
    """Pre-activations Z_l and activations A_l (A_0 = X); the last layer is linear."""
    A = [X]
    Z = []
    for i, (W, b) in enumerate(layers):
        z = A[-1] @ W.T + b
        Z.append(z)
        A.append(silu(z) if i < len(layers) - 1 else z)
    return Z, A


def loss_and_grad(flat_w16, flat_b, sizes, X, t, w=None):
    """MSE loss sum w (y - t)^2 / sum w and its gradient, flat in the parameter layout.

    flat_w16: the parameter vector with weight matrices already rounded to BF16
    (as the device reads them); flat_b: the FP32 master vector, whose bias
    entries are used.
    """
    layers16 = unpack(np.asarray(flat_w16, np.float64), sizes)
    layers32 = unpack(np.asarray(flat_b, np.float64), sizes)
    layers = [(W16, b32) for (W16, _), (_, b32) in zip(layers16, layers32)]
    X = np.asarray(X, np.float64)
    t = np.asarray(t, np.float64)
    w = np.ones_like(t) if w is None else np.asarray(w, np.float64)
    Z, A = forward(layers, X)
    y = A[-1][:, 0]
    tot = w.sum()
    loss = float(np.sum(w * (y - t) ** 2) / tot)
    dz = (2.0 * w * (y - t) / tot)[:, None]
    grads = []
    for i in range(len(layers) - 1, -1, -1):
        W, _ = layers[i]
        dW = dz.T @ A[i]
        db = dz.sum(axis=0)
        grads.append((dW, db))
        if i > 0:
            dz = (dz @ W) * dsilu(Z[i - 1])
    grads.reverse()
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return loss, flat
