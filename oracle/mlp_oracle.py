"""FP64 NumPy oracle of the surrogate MLP -- TEST INFRASTRUCTURE ONLY.

Only tests/ use this module, as the checker of the GPU training kernels (forward, backward,
Adam) and of the tensor-core inference chain. The product never imports it.

Network: x -> [Linear -> GELU] x 4 -> Linear, weights W_l of shape (out, in) (PyTorch Linear
layout), GELU in its tanh form 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3))), loss
mean over rows and outputs of w_o (y - t)^2 with per-output weights w_o.
"""
from __future__ import annotations

import math

import numpy as np

C0 = math.sqrt(2.0 / math.pi)
C1 = 0.044715


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C0 * (x + C1 * x ** 3)))


def gelu_grad(x):
    u = C0 * (x + C1 * x ** 3)
    th = np.tanh(u)
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * C0 * (1.0 + 3.0 * C1 * x * x)


def forward(params, x):
    """params: list of (W, b). Returns (y, cache of pre-activations and inputs)."""
    acts = [x]
    pres = []
    h = x
    for i, (W, b) in enumerate(params):
        z = h @ W.T + b
        pres.append(z)
        h = gelu(z) if i < len(params) - 1 else z
        acts.append(h)
    return h, (acts, pres)


def loss_and_grads(params, x, t, w_out, n_out=None, under=1.0):
    """Loss averaged over rows and the n_out true outputs (padding columns carry w = 0); outputs
    below their target (y < t) weigh ``under`` times more (1: plain weighted MSE)."""
    y, (acts, pres) = forward(params, x)
    n = y.shape[0]
    no = n_out if n_out is not None else y.shape[1]
    r = y - t
    wr = w_out[None, :] * np.where(r < 0.0, under, 1.0)
    loss = float(np.sum(wr * r * r) / (n * no))
    g = 2.0 * wr * r / (n * no)
    grads = [None] * len(params)
    for i in range(len(params) - 1, -1, -1):
        W, b = params[i]
        if i < len(params) - 1:
            g = g * gelu_grad(pres[i])
        grads[i] = (g.T @ acts[i], g.sum(axis=0))
        g = g @ W
    return loss, grads


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    p -= lr * (mh / (np.sqrt(vh) + eps) + wd * p)
