"""FP64 CPU reference of the PI-line initialiser network (TEST INFRASTRUCTURE ONLY).

Used by tests/ to check the CUDA training kernels (ctrecon_b200/csrc/pinet.cu): the same
multilayer perceptron, 3 -> 64 -> 64 -> 64 -> 64 -> 2 with SiLU after each hidden layer, its
mean-squared-error loss and the gradient of that loss with respect to every parameter, in
float64 with numpy.

Parameter vector layout (shared with the CUDA side): for each layer l = 1..5, the weight
matrix W_l[out][in] row-major, then the bias b_l[out].
"""
from __future__ import annotations

import numpy as np

SIZES = [3, 64, 64, 64, 64, 2]


def n_params() -> int:
    return sum(SIZES[i + 1] * SIZES[i] + SIZES[i + 1] for i in range(len(SIZES) - 1))


def unpack(theta: np.ndarray):
    theta = np.asarray(theta, dtype=np.float64)
    out, o = [], 0
    for i in range(len(SIZES) - 1):
        n_in, n_out = SIZES[i], SIZES[i + 1]
        W = theta[o: o + n_out * n_in].reshape(n_out, n_in)
        o += n_out * n_in
        b = theta[o: o + n_out]
        o += n_out
        out.append((W, b))
    assert o == theta.size
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(theta, X):
    """X: (B, 3) features -> (B, 2) outputs and the cached pre-activations."""
    layers = unpack(theta)
    a = np.asarray(X, dtype=np.float64)
    acts, zs = [a], []
    for li, (W, b) in enumerate(layers):
        z = a @ W.T + b
        zs.append(z)
        a = silu(z) if li < len(layers) - 1 else z
        acts.append(a)
    return a, acts, zs


def loss_and_grad(theta, X, Y):
    """Mean over the batch of the squared error summed over the 2 outputs, and its gradient."""
    out, acts, zs = forward(theta, X)
    B = X.shape[0]
    layers = unpack(theta)
    diff = out - Y
    loss = float(np.sum(diff * diff) / B)
    delta = 2.0 * diff / B
    grads = []
    for li in range(len(layers) - 1, -1, -1):
        W, _ = layers[li]
        gW = delta.T @ acts[li]
        gb = delta.sum(axis=0)
        grads.append((gW, gb))
        if li > 0:
            delta = (delta @ W) * dsilu(zs[li - 1])
    grads.reverse()
    g = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, g
