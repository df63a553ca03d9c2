"""CPU oracle of the surrogate MLP -- TEST INFRASTRUCTURE ONLY.

float64 numpy restatement of the network of tomo_shell2026_b200/csrc/tomo_mlp.cu:
[sin y, cos y, sin p, cos p] -> 128 -> 128 -> 128 -> 1, tanh hidden units,
linear output, mean squared error, Adam (beta1 0.9, beta2 0.999, eps 1e-8).
Parameters are one flat vector in the library's layout: per layer the
weights [in][out] row-major, then the biases.  Used only by tests/ to check
the GPU forward pass, gradients and Adam update.
"""
from __future__ import annotations

import numpy as np

DIMS = (4, 128, 128, 128, 1)


def layout():
    off, out = 0, []
    for i in range(4):
        w = (off, DIMS[i], DIMS[i + 1])
        off += DIMS[i] * DIMS[i + 1]
        b = off
        off += DIMS[i + 1]
        out.append((w, b))
    return out, off


def unpack(theta):
    lay, _ = layout()
    th = np.asarray(theta, np.float64)
    Ws, bs = [], []
    for (w0, fi, fo), b0 in lay:
        Ws.append(th[w0:w0 + fi * fo].reshape(fi, fo))
        bs.append(th[b0:b0 + fo])
    return Ws, bs


def forward(theta, x):
    Ws, bs = unpack(theta)
    acts = [np.asarray(x, np.float64)]
    for l in range(4):
        z = acts[-1] @ Ws[l] + bs[l]
        acts.append(np.tanh(z) if l < 3 else z)
    return acts


def loss_and_grad(theta, x, y):
    """Mean squared error and its gradient (flat, library layout)."""
    Ws, _ = unpack(theta)
    acts = forward(theta, x)
    n = acts[0].shape[0]
    yhat = acts[-1][:, 0]
    d = yhat - np.asarray(y, np.float64)
    loss = float(np.mean(d * d))
    dz = (2.0 * d / n)[:, None]
    grads_w, grads_b = [None] * 4, [None] * 4
    for l in range(3, -1, -1):
        grads_w[l] = acts[l].T @ dz
        grads_b[l] = dz.sum(0)
        if l > 0:
            dz = (dz @ Ws[l].T) * (1.0 - acts[l] ** 2)
    lay, total = layout()
    g = np.zeros(total)
    for l, ((w0, fi, fo), b0) in enumerate(lay):
        g[w0:w0 + fi * fo] = grads_w[l].ravel()
        g[b0:b0 + fo] = grads_b[l]
    return loss, g


def adam_step(theta, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update at step t (1-based); returns (theta, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v


def features(ypr):
    y, p = np.asarray(ypr, np.float32)[:, 0], np.asarray(ypr, np.float32)[:, 1]
    return np.stack([np.sin(y), np.cos(y), np.sin(p), np.cos(p)], 1).astype(np.float32)
