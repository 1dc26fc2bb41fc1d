"""CPU oracle of the selector MLP -- TEST INFRASTRUCTURE ONLY.

numpy (float64) restatement of the network the CUDA kernels train
(rw-spgemm_b200/csrc/tsg_mlp.cu): F -> H -> H -> O with ReLU, masked mean
squared error, parameters packed as W1[F][H] b1 W2[H][H] b2 W3[H][O] b3.
Used to check the GPU gradients and the Adam update.
"""
import numpy as np


def unpack(w, F, H, O):
    o = 0
    out = []
    for shape in ((F, H), (H,), (H, H), (H,), (H, O), (O,)):
        n = int(np.prod(shape))
        out.append(np.asarray(w[o:o + n], dtype=np.float64).reshape(shape))
        o += n
    return out


def forward(w, X, F, H, O):
    W1, b1, W2, b2, W3, b3 = unpack(w, F, H, O)
    h1 = np.maximum(X @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h1, h2, h2 @ W3 + b3


def loss_and_grads(w, X, T, M, F, H, O):
    X = np.asarray(X, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w, F, H, O)
    h1, h2, y = forward(w, X, F, H, O)
    M = np.ones_like(y) if M is None else np.asarray(M, np.float64)
    den = max(M.sum(), 1.0)
    r = y - T
    loss = float((M * r * r).sum() / den)
    dy = 2 * M * r / den
    gW3, gb3 = h2.T @ dy, dy.sum(0)
    d2 = (dy @ W3.T) * (h2 > 0)
    gW2, gb2 = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    gW1, gb1 = X.T @ d1, d1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g


def adam(w, g, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    w = w - lr * (m1 / (1 - b1 ** step)) / (np.sqrt(m2 / (1 - b2 ** step)) + eps)
    return w, m1, m2
