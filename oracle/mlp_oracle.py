"""ORACLE — test infrastructure only: the scheduler network restated in FP64 numpy
(forward, mean-squared-error loss and its gradient) to check the CUDA kernels of
starplat_b200/csrc/sp_mlp.cu. Parameter layout: W1 (H x IN), b1, W2 (H x H), b2, w3, b3."""
import numpy as np

IN, H = 13, 32


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + H * IN].reshape(H, IN); o += H * IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ w3 + b3, h1, h2


def loss_grad(p, X, T):
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, h1, h2 = forward(p, X)
    N = X.shape[0]
    r = y - T
    L = float((r * r).mean())
    gy = 2.0 * r / N
    gw3 = h2.T @ gy
    gb3 = gy.sum()
    dz2 = np.outer(gy, w3) * (1 - h2 * h2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (1 - h1 * h1)
    gW1 = dz1.T @ X
    gb1 = dz1.sum(0)
    return L, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
