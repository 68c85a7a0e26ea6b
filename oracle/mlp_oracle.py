"""CPU oracle of the plan cost model's network (TEST INFRASTRUCTURE ONLY).

Float64 numpy restatement of the engine's 24 -> 64 -> 64 -> 1 ReLU MLP
(cuda_fot_b200/csrc/mlp.cu): the same parameter layout
W1[IN][H] | b1[H] | W2[H][H] | b2[H] | W3[H] | b3, inputs standardised by
mean / std, loss 0.5/N * sum (y - t)^2.  Gives the analytic gradient the GPU
backward kernels are checked against, and a central finite-difference
gradient that checks the analytic one.
"""
import numpy as np

IN, H = 24, 64


def split(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + IN * H].reshape(IN, H); o += IN * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def n_params():
    return IN * H + H + H * H + H + H + 1


def forward(p, X, mean, std):
    W1, b1, W2, b2, W3, b3 = split(p)
    x = (np.asarray(X, np.float64) - mean) / std
    a1 = x @ W1 + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0)
    y = h2 @ W3 + b3
    return y, (x, a1, h1, a2, h2)


def loss(p, X, t, mean, std):
    y, _ = forward(p, X, mean, std)
    r = y - t
    return 0.5 * np.mean(r * r)


def grad(p, X, t, mean, std):
    W1, b1, W2, b2, W3, b3 = split(p)
    y, (x, a1, h1, a2, h2) = forward(p, X, mean, std)
    n = X.shape[0]
    dy = (y - t) / n
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    d2 = np.outer(dy, W3) * (a2 > 0)
    gW2 = h1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (a1 > 0)
    gW1 = x.T @ d1
    gb1 = d1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])


def fd_grad(p, X, t, mean, std, idx, h=1e-6):
    p = np.asarray(p, np.float64)
    out = []
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        out.append((loss(p + e, X, t, mean, std) - loss(p - e, X, t, mean, std)) / (2 * h))
    return np.array(out)
