"""CPU checks of the FP64 cache oracle itself (oracle/nrc_oracle.py):
back-propagated gradients against central finite differences, and BF16
rounding."""

import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "oracle"))
import nrc_oracle as no  # noqa: E402


def _batch(n, seed=0):
    rng = np.random.default_rng(seed)
    feats = rng.uniform(0, 1, (n, 64))
    feats[:, 50:] = 0
    targets = rng.uniform(0, 2, (n, 4))
    return feats, targets


def test_gradient_matches_finite_differences():
    w = no.xavier(3) * 1.5
    feats, targets = _batch(64)
    loss, g = no.loss_grad(w, feats, targets, bf=False)
    rng = np.random.default_rng(5)
    idx = list(rng.choice(5 * no.SQ, 40, replace=False)) + \
        list(5 * no.SQ + rng.choice(3 * 64, 10, replace=False))
    for i in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        lp, _ = no.loss_grad(wp, feats, targets, bf=False)
        lm, _ = no.loss_grad(wm, feats, targets, bf=False)
        # the loss detaches y in the denominator: compare with the
        # gradient of the same detached objective
        fd = _detached_fd(w, feats, targets, i, h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


def _detached_fd(w, feats, targets, i, h):
    _, y0 = no.forward(w, feats, bf=False)
    den = y0 * y0 + 0.01
    t = targets[:, :3]

    def obj(ww):
        _, y = no.forward(ww, feats, bf=False)
        return np.sum((y - t) ** 2 / den) / (3.0 * len(feats))
    wp, wm = w.copy(), w.copy()
    wp[i] += h
    wm[i] -= h
    return (obj(wp) - obj(wm)) / (2 * h)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, 3.14159265, -2.5e-3])
    r = no.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0078125
    assert abs(r[3] - 3.140625) < 1e-12
    assert abs(r[4] + 2.5e-3) < 1e-5


def test_adam_moves_against_gradient():
    w = no.xavier(1)
    g = np.sign(np.random.default_rng(0).normal(size=no.NPARAMS))
    g[5 * no.SQ + 3 * 64:] = 0
    w2, m, v = no.adam(w, np.zeros_like(w), np.zeros_like(w), g, 1)
    d = (w2 - w)[g != 0]
    assert np.allclose(d, -1e-2 * np.sign(g[g != 0]), rtol=1e-6)


def test_grid_features_and_gradient_are_adjoint():
    """The hash grid's features are linear in the table and grid_grad is
    their adjoint: <grid_grad(x, d), T> = sum d * features(T, x); the
    trilinear weights of a cell sum to 1, and a constant table gives that
    constant as every feature."""
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, (500, 3)).astype(np.float32)
    x[:5] = [[0, 0, 0], [1, 1, 1], [1, 0, 0.5], [0.5, 1, 0], [1e-7, 1, 1]]
    T = rng.normal(size=no.GRID_PARAMS)
    d = rng.normal(size=(len(x), 16))
    lhs = np.dot(no.grid_grad(x, d), T)
    rhs = np.sum(d * no.grid_features(T, x))
    assert abs(lhs - rhs) <= 1e-9 * abs(rhs)
    for l in range(no.GRID_LEVELS):
        idx, wt = no.grid_corners(x, l)
        assert np.allclose(wt.sum(1), 1.0)
        assert idx.min() >= l * no.GRID_T and idx.max() < (l + 1) * no.GRID_T
    f = no.grid_features(np.full(no.GRID_PARAMS, 0.25), x)
    assert np.allclose(f, 0.25)
    # dense levels: distinct corners get distinct entries
    idx, _ = no.grid_corners(np.array([[0.3, 0.6, 0.9]], np.float32), 0)
    assert len(set(idx[0])) == 8
