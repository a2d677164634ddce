"""CPU restatement of the rule-picking network's forward and backward pass.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of libtce's
tce_mlp_loss_grad (forward, sigmoid cross-entropy, backward).  The product
never imports it.  The network has no counterpart in the reference (its
t-quadrature uses one fixed rule per run, precompute_t.f90:5-14); this file
states the textbook computation in float64:

    x  = (X - mu) / sig
    h1 = relu(x W1^T + b1),  h2 = relu(h1 W2^T + b2),  z = h2 W3^T + b3
    L  = mean_r sum_c [ max(z,0) - z Y + log(1 + exp(-|z|)) ]

Parameters flat: W1[nh][nf] b1[nh] W2[nh][nh] b2[nh] W3[nc][nh] b3[nc].
"""
from __future__ import annotations

import numpy as np


def unpack(p, nf, nh, nc):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((nh, nf), (nh,), (nh, nh), (nh,), (nc, nh), (nc,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    assert o == len(p)
    return out


def forward(p, mu, sig, X, nf, nh, nc):
    W1, b1, W2, b2, W3, b3 = unpack(p, nf, nh, nc)
    x = (np.asarray(X, np.float64) - mu) / sig
    h1 = np.maximum(x @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return x, h1, h2, h2 @ W3.T + b3


def loss_grad(p, mu, sig, X, Y, nf, nh, nc):
    W1, b1, W2, b2, W3, b3 = unpack(p, nf, nh, nc)
    x, h1, h2, z = forward(p, mu, sig, X, nf, nh, nc)
    Y = np.asarray(Y, np.float64)
    B = len(Y)
    loss = float(np.mean(np.sum(np.maximum(z, 0) - z * Y + np.log1p(np.exp(-np.abs(z))), axis=1)))
    dz = (1.0 / (1.0 + np.exp(-z)) - Y) / B
    gW3, gb3 = dz.T @ h2, dz.sum(0)
    dh2 = (dz @ W3) * (h2 > 0)
    gW2, gb2 = dh2.T @ h1, dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    gW1, gb1 = dh1.T @ x, dh1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])


def predict(p, mu, sig, X, nf, nh, nc):
    return 1.0 / (1.0 + np.exp(-forward(p, mu, sig, X, nf, nh, nc)[3]))
