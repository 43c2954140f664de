"""NumPy float64 restatement of the estimator MLP (test infrastructure only).

Network: x (16) -> ReLU(x W1 + b1) (64) -> ReLU(h1 W2 + b2) (64) -> h2 W3 + b3 (2),
loss = 1/(2m) * sum over samples and outputs of (y - t)^2.  Parameters are one
flat vector in the engine's layout: W1[16x64], b1[64], W2[64x64], b2[64],
W3[64x2], b3[2], row-major with the input index first.
"""
import numpy as np

F, H, O = 16, 64, 2


def unpack(w):
    w = np.asarray(w, np.float64)
    o = 0
    out = []
    for shape in ((F, H), (H,), (H, H), (H,), (H, O), (O,)):
        sz = int(np.prod(shape))
        out.append(w[o:o + sz].reshape(shape))
        o += sz
    assert o == w.size
    return out


def forward(x, w):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z1 = x @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3 + b3


def loss_grad(x, t, w):
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(w)
    m = x.shape[0]
    z1 = x @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ W3 + b3
    e = y - t
    loss = 0.5 * np.sum(e * e) / m
    dy = e / m
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    d2 = (dy @ W3.T) * (z2 > 0)
    gW2 = h1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (z1 > 0)
    gW1 = x.T @ d1
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
