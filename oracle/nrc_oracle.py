"""Test infrastructure only: FP64 oracle of the neural radiance cache.

The reference renderer has no learned component, so there is nothing to
restate; this is an independent numpy implementation of the network the GPU
kernels implement (64 -> 5 x 64 ReLU -> 3, no biases, weights [out][in]),
its relative L2 loss, gradients and Adam step, plus the input encoding.
`bf16=True` rounds to BF16 at the points the tensor-core kernels do
(weights, layer inputs, output-gradient and back-propagated gradients), so
the GPU can be compared tightly; `bf16=False` is plain FP64, used for the
finite-difference check of the gradients themselves.
"""

import numpy as np

SQ = 4096
NPARAMS = 5 * SQ + 8 * 64


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(w):
    """Split the flat parameter vector into 6 matrices [out][in]."""
    w = np.asarray(w, np.float64)
    mats = [w[l * SQ:(l + 1) * SQ].reshape(64, 64) for l in range(5)]
    mats.append(w[5 * SQ:5 * SQ + 8 * 64].reshape(8, 64)[:3])
    return mats


def forward(w, feats, bf=True):
    """Layer inputs a_0..a_5 and outputs y (n x 3)."""
    rnd = bf16 if bf else (lambda x: np.asarray(x, np.float64))
    W = [rnd(m) for m in layers(w)]
    a = [rnd(feats)]
    for l in range(5):
        z = a[-1] @ W[l].T
        a.append(rnd(np.maximum(z, 0.0)))
    y = a[-1] @ W[5].T
    return a, y


def loss_grad(w, feats, targets, bf=True):
    """Loss mean((y - t)^2 / (y^2 + 0.01)) and its gradient (flat, the
    layout of the parameter vector; padded output rows zero)."""
    rnd = bf16 if bf else (lambda x: np.asarray(x, np.float64))
    W = [rnd(m) for m in layers(w)]
    a, y = forward(w, feats, bf)
    n = len(feats)
    t = np.asarray(targets, np.float64)[:, :3]
    den = y * y + 0.01
    loss = np.sum((y - t) ** 2 / den) / (3.0 * n)
    dz = rnd(2.0 * (y - t) / den / (3.0 * n))
    g = np.zeros(NPARAMS)
    for l in range(5, -1, -1):
        dW = dz.T @ a[l]
        if l == 5:
            g[5 * SQ:5 * SQ + 3 * 64] = dW.ravel()
        else:
            g[l * SQ:(l + 1) * SQ] = dW.ravel()
        if l == 0:
            break
        dA = dz @ W[l]
        dz = rnd(dA * (a[l] > 0))
    return loss, g


def adam(w, m, v, g, step, lr=1e-2, b1=0.9, b2=0.99, eps=1e-15):
    """One Adam step (the padded output rows stay zero)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    w = w - lr * mh / (np.sqrt(vh) + eps)
    w[5 * SQ + 3 * 64:] = 0.0
    return w, m, v


def encode(raw, lo, hi):
    """12 raw inputs per query -> 64 features (FP64)."""
    raw = np.asarray(raw, np.float64)
    n = len(raw)
    f = np.zeros((n, 64))
    x = np.clip((raw[:, :3] - lo) / (hi - lo), 0.0, 1.0)
    for a in range(3):
        for k in range(6):
            ang = np.pi * (2.0 ** k) * x[:, a]
            f[:, a * 12 + 2 * k] = np.sin(ang)
            f[:, a * 12 + 2 * k + 1] = np.cos(ang)
    d = raw[:, 3:6]
    th = np.arccos(np.clip(d[:, 2], -1, 1)) / np.pi
    ph = np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi) + 0.5
    for j, u in enumerate((th, ph)):
        for k in range(2):
            ang = np.pi * (2.0 ** k) * u
            f[:, 36 + j * 4 + 2 * k] = np.sin(ang)
            f[:, 36 + j * 4 + 2 * k + 1] = np.cos(ang)
    f[:, 44:47] = 0.5 * (raw[:, 6:9] + 1.0)
    f[:, 47:50] = raw[:, 9:12]
    return f


def xavier(seed=1):
    """A deterministic starting point for CPU-only checks."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAMS)
    for l in range(6):
        nout = 3 if l == 5 else 64
        b = np.sqrt(6.0 / (64 + nout))
        blk = rng.uniform(-b, b, (nout, 64))
        if l == 5:
            w[5 * SQ:5 * SQ + 3 * 64] = blk.ravel()
        else:
            w[l * SQ:(l + 1) * SQ] = blk.ravel()
    return w
