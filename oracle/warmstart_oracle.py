"""Oracle of the learned warm start's network (test infrastructure only: imported by tests/,
never by the library).

A NumPy restatement, in FP64, of what the library's kernels compute (csrc/warmstart.cu): the
forward pass H = W1 X, Y = W2 H of the two-layer linear network, the loss
sum (Y - T)^2 / batch and its gradients dW2 = dY H^T, dW1 = W2^T dY X^T with dY = 2 (Y - T) / batch,
and one bias-corrected Adam step. The GPU kernels run in FP32 and are checked against these.
"""
from __future__ import annotations

import numpy as np


def forward(W1, W2, X):
    H = W1.astype(np.float64) @ X.astype(np.float64)
    return H, W2.astype(np.float64) @ H


def loss_and_grads(W1, W2, X, T):
    X = X.astype(np.float64)
    H, Y = forward(W1, W2, X)
    batch = X.shape[1]
    D = Y - T.astype(np.float64)
    dY = 2.0 * D / batch
    dW2 = dY @ H.T
    dW1 = (W2.astype(np.float64).T @ dY) @ X.T
    return float(np.sum(D * D) / batch), dW1, dW2


def adam_step(p, g, m, v, lr, step, beta1=0.9, beta2=0.999, eps=1e-8):
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mhat = m / (1 - beta1 ** step)
    vhat = v / (1 - beta2 ** step)
    return p - lr * mhat / (np.sqrt(vhat) + eps), m, v
