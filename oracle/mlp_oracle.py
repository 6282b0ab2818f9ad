"""CPU oracle for the learned scheduler's MLP: TEST INFRASTRUCTURE ONLY.

float64 numpy restatement of the network in custingeralg_b200/csrc/tc_mlp.cu (same parameter
layout): features -> 64 -> 64 -> TC_MLP_OUT with ReLU, loss = mean_i (y_i[s_i] - label_i)^2.
Used to check the GPU forward pass and gradients.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 4, 64, 3


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + HID * IN].reshape(HID, IN); o += HID * IN
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + OUT * HID].reshape(OUT, HID); o += OUT * HID
    b3 = p[o:o + OUT]; o += OUT
    assert o == p.size
    return W1, b1, W2, b2, W3, b3


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3.T + b3
    return y, (X, a1, h1, a2, h2)


def loss_and_grad(p, X, strat, label):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    y, (X, a1, h1, a2, h2) = forward(p, X)
    n = X.shape[0]
    idx = np.arange(n)
    d = y[idx, strat] - np.asarray(label, dtype=np.float64)
    loss = float(np.mean(d * d))
    gy = np.zeros_like(y)
    gy[idx, strat] = 2.0 * d / n
    gW3 = gy.T @ h2
    gb3 = gy.sum(0)
    g2 = (gy @ W3) * (a2 > 0)
    gW2 = g2.T @ h1
    gb2 = g2.sum(0)
    g1 = (g2 @ W2) * (a1 > 0)
    gW1 = g1.T @ X
    gb1 = g1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, grad
