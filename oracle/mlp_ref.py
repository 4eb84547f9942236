"""CPU reference of the shell-proposal MLP (test infrastructure).

float64 numpy restatement of the network the library trains on the GPU:
126 -> 64 (SiLU) -> 64 (SiLU) -> 8, softmax cross-entropy averaged over the
batch, Adam (beta1 0.9, beta2 0.999, eps 1e-8). Parameter layout: W1[64][126]
b1[64] W2[64][64] b2[64] W3[8][64] b3[8]. The tests check the GPU forward,
gradient and Adam kernels against it, and it against finite differences.
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 126, 64, 8
SHAPES = [(N_HID, N_IN), (N_HID,), (N_HID, N_HID), (N_HID,), (N_OUT, N_HID), (N_OUT,)]


def unpack(p):
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(p[o:o + n], dtype=np.float64).reshape(s))
        o += n
    return out


def pack(parts):
    return np.concatenate([np.asarray(x).reshape(-1) for x in parts])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1.T + b1
    h1 = z1 * _sig(z1)
    z2 = h1 @ W2.T + b2
    h2 = z2 * _sig(z2)
    z3 = h2 @ W3.T + b3
    z3s = z3 - z3.max(axis=1, keepdims=True)
    e = np.exp(z3s)
    probs = e / e.sum(axis=1, keepdims=True)
    return dict(z1=z1, h1=h1, z2=z2, h2=h2, z3=z3, probs=probs)


def loss_and_grad(p, X, y):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(y)
    B = X.shape[0]
    f = forward(p, X)
    probs = f["probs"]
    loss = -np.mean(np.log(probs[np.arange(B), y]))
    dz3 = probs.copy()
    dz3[np.arange(B), y] -= 1.0
    dz3 /= B
    gW3 = dz3.T @ f["h2"]
    gb3 = dz3.sum(0)
    dh2 = dz3 @ W3
    s2 = _sig(f["z2"])
    dz2 = dh2 * s2 * (1.0 + f["z2"] * (1.0 - s2))
    gW2 = dz2.T @ f["h1"]
    gb2 = dz2.sum(0)
    dh1 = dz2 @ W2
    s1 = _sig(f["z1"])
    dz1 = dh1 * s1 * (1.0 + f["z1"] * (1.0 - s1))
    gW1 = dz1.T @ X
    gb1 = dz1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3])


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1 = 1 - b1 ** step
    c2 = 1 - b2 ** step
    p = p - lr * (m / c1) / (np.sqrt(v / c2) + eps)
    return p, m, v
