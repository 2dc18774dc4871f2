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


# Multiresolution hash grid of the position (Mueller, Evans, Schied and
# Keller 2022): levels of GRID_T entries of 2 features, GRID_RES cells per
# axis over the unit box; corners indexed densely where (res + 1)^3 fits a
# level's table, else by the spatial hash of Teschner et al. 2003.
GRID_LEVELS = 8
GRID_T = 1 << 17
GRID_RES = (16, 28, 52, 95, 172, 312, 565, 1024)
GRID_PARAMS = GRID_LEVELS * GRID_T * 2


def unit_position(raw, lo, hi):
    """Positions in the unit box as the device computes them: FP32
    (p - lo) * (1 / (hi - lo)), clamped to [0, 1]."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    inv = np.where(hi > lo, np.float32(1.0) / (hi - lo), np.float32(1.0))
    p = np.asarray(raw, np.float32)[:, :3]
    return np.clip((p - lo) * inv.astype(np.float32), 0.0, 1.0).astype(
        np.float32)


def grid_index(l, x, y, z, scene=0):
    """Table entry of lattice corners (x, y, z) (uint32 arrays) of level l."""
    r1 = np.uint32(GRID_RES[l] + 1)
    x, y, z = (np.asarray(v, np.uint32) for v in (x, y, z))
    with np.errstate(over="ignore"):
        if scene == 0 and int(r1) ** 3 <= GRID_T:
            i = x + r1 * (y + r1 * z)
        else:
            i = (x ^ (y * np.uint32(2654435761)) ^ (z * np.uint32(805459861))
                 ^ np.uint32((scene * 0x9e3779b9) & 0xffffffff))
    return (i & np.uint32(GRID_T - 1)).astype(np.int64) + l * GRID_T


def grid_corners(x, l):
    """Per level-l cell corner b (0..7): entry indices (n, 8) and trilinear
    weights (n, 8), FP32 cell arithmetic as on the device."""
    res = GRID_RES[l]
    p = (x.astype(np.float32) * np.float32(res)).astype(np.float32)
    c = np.minimum(np.floor(p), res - 1).astype(np.uint32)
    w = (p - c.astype(np.float32)).astype(np.float64)
    idx = np.zeros((len(x), 8), np.int64)
    wt = np.ones((len(x), 8))
    for b in range(8):
        o = [(b >> a) & 1 for a in range(3)]
        idx[:, b] = grid_index(l, c[:, 0] + o[0], c[:, 1] + o[1],
                               c[:, 2] + o[2])
        for a in range(3):
            wt[:, b] *= w[:, a] if o[a] else 1.0 - w[:, a]
    return idx, wt


def grid_features(table, x):
    """(n, 2 GRID_LEVELS) features of unit-box positions x."""
    t = np.asarray(table, np.float64).reshape(-1, 2)
    f = np.zeros((len(x), 2 * GRID_LEVELS))
    for l in range(GRID_LEVELS):
        idx, wt = grid_corners(x, l)
        f[:, 2 * l:2 * l + 2] = np.einsum("nb,nbk->nk", wt, t[idx])
    return f


def grid_grad(x, dfeat):
    """Gradient of the table given d loss / d feature (n, 2 GRID_LEVELS)."""
    g = np.zeros((GRID_PARAMS // 2, 2))
    for l in range(GRID_LEVELS):
        idx, wt = grid_corners(x, l)
        for k in range(2):
            np.add.at(g[:, k], idx.ravel(),
                      (wt * dfeat[:, 2 * l + k:2 * l + k + 1]).ravel())
    return g.ravel()


def encode(raw, lo, hi, table=None):
    """12 raw inputs per query -> 64 features (FP64): 0..15 hash grid (zero
    without a table), 16..33 sin/cos(2^k pi x), k = 0..2, per axis, 34..41
    direction, 42..44 normal, 45..47 albedo."""
    raw = np.asarray(raw, np.float64)
    n = len(raw)
    f = np.zeros((n, 64))
    x = unit_position(raw, lo, hi)
    if table is not None:
        f[:, :16] = grid_features(table, x)
    xd = x.astype(np.float64)
    for a in range(3):
        for k in range(3):
            ang = np.pi * (2.0 ** k) * xd[:, a]
            f[:, 16 + a * 6 + 2 * k] = np.sin(ang)
            f[:, 16 + a * 6 + 2 * k + 1] = np.cos(ang)
    d = raw[:, 3:6]
    th = np.arccos(np.clip(d[:, 2], -1, 1)) / np.pi
    ph = np.arctan2(d[:, 1], d[:, 0]) / (2 * np.pi) + 0.5
    for j, u in enumerate((th, ph)):
        for k in range(2):
            ang = np.pi * (2.0 ** k) * u
            f[:, 34 + j * 4 + 2 * k] = np.sin(ang)
            f[:, 34 + j * 4 + 2 * k + 1] = np.cos(ang)
    f[:, 42:45] = 0.5 * (raw[:, 6:9] + 1.0)
    f[:, 45:48] = raw[:, 9:12]
    return f


def feature_grad(w, feats, targets, bf=True):
    """d loss / d feature (n, 64) of the loss of loss_grad: dz_0 W_0 with
    dz_0 as the backward pass leaves it (BF16-rounded with bf)."""
    rnd = bf16 if bf else (lambda x: np.asarray(x, np.float64))
    W = [rnd(m) for m in layers(w)]
    a, y = forward(w, feats, bf)
    n = len(feats)
    t = np.asarray(targets, np.float64)[:, :3]
    dz = rnd(2.0 * (y - t) / (y * y + 0.01) / (3.0 * n))
    for l in range(5, 0, -1):
        dz = rnd((dz @ W[l]) * (a[l] > 0))
    return dz @ W[0]


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
