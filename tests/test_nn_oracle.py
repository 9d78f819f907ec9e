"""The NumPy restatement of the learned-guess model: its analytic gradient against finite differences (no GPU)."""

import numpy as np

import nn_oracle as N


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0])
    r = N.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0


def test_exact_gradient_equals_finite_differences():
    rng = np.random.default_rng(0)
    n = 40
    flat = rng.normal(scale=0.3, size=7328)
    inv = rng.normal(size=(n, N.N_IN))
    vec = rng.normal(scale=0.02, size=(n, N.N_CH, 3))
    tgt = rng.normal(scale=0.02, size=(n, 3))
    loss, g = N.loss_grad(flat, inv, vec, tgt, 1.0 / (n * 0.02**2), rounded=False)
    h = 1e-6
    for k in rng.choice(flat.size, 25, replace=False):
        d = np.zeros_like(flat)
        d[k] = h
        lp = N.loss_grad(flat + d, inv, vec, tgt, 1.0 / (n * 0.02**2), rounded=False)[0]
        lm = N.loss_grad(flat - d, inv, vec, tgt, 1.0 / (n * 0.02**2), rounded=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_mpnn_oracle_gradient_equals_central_differences():
    """The message-passing model's analytic gradient (unrounded) against central differences."""
    rng = np.random.default_rng(4)
    n, ne = 40, 300
    src = rng.integers(0, n, ne)
    dst = (src + 1 + rng.integers(0, n - 1, ne)) % n
    src, dst = np.concatenate([src, dst]), np.concatenate([dst, src])  # symmetric graph
    d = np.concatenate([rng.uniform(0.1, 0.5, ne)] * 2)
    phi = N.radial(d, 0.5)
    inv = rng.normal(size=(n, N.N_IN))
    vec = rng.normal(scale=0.01, size=(n, N.N_CH, 3))
    tgt = rng.normal(scale=1e-4, size=(n, 3))
    w = rng.normal(scale=0.2, size=N.mpnn_nparam())
    loss, g = N.mpnn_loss_grad(w, inv, vec, src, dst, phi, tgt, 2e-4, 1e6, rounded=False)
    h = 1e-6
    bounds = np.cumsum([0] + [int(np.prod(sh)) for sh in N.MPNN_SHAPES])
    every_block = [int(rng.integers(lo, hi)) for lo, hi in zip(bounds[:-1], bounds[1:])]
    for k in every_block + list(rng.choice(w.size, 10, replace=False)):
        e = np.zeros_like(w)
        e[k] = h
        lp = N.mpnn_loss_grad(w + e, inv, vec, src, dst, phi, tgt, 2e-4, 1e6, rounded=False)[0]
        lm = N.mpnn_loss_grad(w - e, inv, vec, src, dst, phi, tgt, 2e-4, 1e6, rounded=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1e-3, abs(fd)), (k, fd, g[k])
