"""CPU oracle of the sifter MLP (test infrastructure): numpy float64 forward and backward passes of
the 1728 -> 256 -> 128 -> 1 ReLU network on the mean binary cross-entropy, with the GPU kernels'
bf16 rounding points emulated (round-to-nearest-even to bf16 of: the fp16 patches, the weights, the
ReLU activations, and of the loss gradients where they enter a product), and a plain float64 version
for finite-difference checks of the backward formulas. It is the checker of the CUDA kernels in
pirate_b200/csrc/sifter.cu, never part of the product."""

import numpy as np

SHAPES = [(256, 1728), (256,), (128, 256), (128,), (1, 128), (1,)]


def split(p):
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(p[o:o + n], dtype=np.float64).reshape(s))
        o += n
    return out


def bf16(x):
    """Rounds to the nearest bfloat16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7fff + ((u >> 16) & 1)) & 0xffff0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _loss(z, y):
    return np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))


def forward(p, x, emulate=True):
    """Logits and intermediates. x: (n, 1728) patches (fp16 values)."""
    W1, b1, W2, b2, W3, b3 = split(p)
    r = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    X = r(np.asarray(x, dtype=np.float32))
    z1 = X @ r(W1).T + b1
    h1 = r(np.maximum(z1, 0))
    z2 = h1 @ r(W2).T + b2
    h2 = r(np.maximum(z2, 0))
    z3 = (h2 @ r(W3).T + b3)[:, 0]
    return z3, dict(X=X, z1=z1, h1=h1, z2=z2, h2=h2, z3=z3)


def gradients(p, x, y, emulate=True):
    """(loss, flat gradient) of the mean binary cross-entropy, in the GPU's order of operations."""
    W1, b1, W2, b2, W3, b3 = split(p)
    r = bf16 if emulate else (lambda v: np.asarray(v, dtype=np.float64))
    y = np.asarray(y, dtype=np.float64)
    z3, c = forward(p, x, emulate)
    n = len(y)
    g = (1.0 / (1.0 + np.exp(-z3)) - y) / n
    if emulate:
        g = g.astype(np.float32).astype(np.float64)
    gr = r(g)
    dW3 = (gr @ c["h2"])[None, :]
    db3 = np.array([g.sum()])
    gH2 = np.outer(gr, r(W3)[0])
    g2 = gH2 * (c["z2"] > 0)
    g2r = r(g2)
    dW2 = g2r.T @ c["h1"]
    db2 = g2.sum(axis=0)
    gH1 = g2r @ r(W2)
    g1 = gH1 * (c["z1"] > 0)
    dW1 = r(g1).T @ c["X"]
    db1 = g1.sum(axis=0)
    grad = np.concatenate([a.ravel() for a in (dW1, db1, dW2, db2, dW3, db3)])
    return _loss(z3, y), grad


def loss(p, x, y):
    z3, _ = forward(p, x, emulate=False)
    return _loss(z3, np.asarray(y, dtype=np.float64))
