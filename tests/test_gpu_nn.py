"""The learned initial guess on the GPU: tensor-core kernels against the NumPy model, equivariance
of the features, and what a trained model gains over the untrained (linear extrapolation) guess."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

import nn_oracle as N  # noqa: E402


def _dev(a, dt=torch.float32):
    return torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def test_tensor_core_gradient_matches_numpy():
    """Forward and the weight gradient of the BF16 WMMA kernels equal the NumPy model rounded at the same points."""
    from pgm_jax_b200.learned import GuessModel, init_weights

    rng = np.random.default_rng(1)
    n = 300  # not a multiple of the 64-sample tile
    w = init_weights(3) + rng.normal(scale=0.05, size=7328).astype(np.float32)
    inv = rng.normal(size=(n, N.N_IN)).astype(np.float32)
    vec = rng.normal(scale=0.02, size=(n, N.N_CH, 3)).astype(np.float32)
    tgt = rng.normal(scale=0.02, size=(n, 3)).astype(np.float32)
    m = GuessModel(w)
    mu = m.predict(_dev(inv), _dev(vec)).cpu().numpy()
    mu_ref, _ = N.forward(w, inv, vec)
    assert np.abs(mu - mu_ref).max() <= 1e-4 * np.abs(mu_ref).max()
    scale = 1.0 / (n * 0.02**2)
    loss = m.loss_grad(_dev(inv), _dev(vec), _dev(tgt), scale)
    g = m.g.cpu().numpy()
    loss_ref, g_ref = N.loss_grad(w, inv, vec, tgt, scale)
    assert abs(loss - loss_ref) <= 1e-4 * loss_ref
    assert np.linalg.norm(g - g_ref) <= 2e-3 * np.linalg.norm(g_ref), np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    # and close to the exact (unrounded) gradient: BF16 is the only approximation
    _, g_ex = N.loss_grad(w, inv, vec, tgt, scale, rounded=False)
    assert np.linalg.norm(g - g_ex) <= 5e-2 * np.linalg.norm(g_ex)


def test_features_turn_with_the_system():
    """A 90-degree turn of a cubic box: invariants unchanged, vector channels turned."""
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.learned import features
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(4, 1.25, seed=4)
    st = MDSettings(precision="double", cutoff=0.6, ewald_beta=6.0, pme_grid=(32, 32, 32))
    ff = PGMForceField(s, H, st)
    rng = np.random.default_rng(2)
    hist = rng.normal(scale=0.01, size=(4, s.n, 3))
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    pos_r = (pos @ R.T) % 1.25
    inv0, vec0, b0 = features(ff, _dev(pos, torch.float64), _dev(H[None], torch.float64), _dev(hist, torch.float64))
    inv1, vec1, b1 = features(ff, _dev(pos_r, torch.float64), _dev(H[None], torch.float64), _dev(hist @ R.T, torch.float64))
    assert np.abs(b0.cpu().numpy() @ R.T - b1.cpu().numpy()).max() <= 1e-8 * float(b0.abs().max())
    inv0, inv1 = inv0.cpu().numpy(), inv1.cpu().numpy()
    assert np.abs(inv0 - inv1).max() <= 1e-4 * max(1.0, np.abs(inv0).max())
    v0, v1 = vec0.cpu().numpy(), vec1.cpu().numpy()
    assert np.abs(v0 @ R.T - v1).max() <= 1e-4 * np.abs(v0).max()


def test_trained_guess_beats_extrapolation_and_solves_to_tolerance():
    """Plain-solver MD writes (features, converged dipoles); a few hundred GPU Adam steps train the
    model; on later frames its guess is closer than 2 mu1 - mu2, and MD started from it converges to
    the same tolerance."""
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.learned import GuessModel, collect, guess_errors
    from pgm_jax_b200.md import RigidMD
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(5, 1.55, seed=6)
    kw = dict(precision="mixed", cutoff=0.7, ewald_beta=5.0, pme_grid=(32, 32, 32), dipole_tol=1e-6, max_iter=100)
    ff = PGMForceField(s, H, MDSettings(predictor="nn", **kw))
    md = RigidMD(ff, pos, H, temperature=300.0, dt_fs=1.0, gamma_ps=5.0, seed=2)
    train = collect(md, 60)
    held = collect(md, 12)
    model = GuessModel(seed=0)
    before = guess_errors(model, held)
    model.train(train, iters=800, batch=8192, lr=2e-3)
    after = guess_errors(model, held)
    assert abs(before["model"] - before["linear"]) <= 1e-3 * before["linear"]  # untrained = extrapolation
    assert after["model"] < 0.97 * before["linear"], (before, after)  # the trained model gains on unseen frames
    model.install(ff)
    its = []
    for _ in range(8):
        md.step()
        its.append(int(ff._iters[0]))
        assert float(ff._resid[0]) <= 1e-6 and not int(ff._status[0]) & 0x2
    assert np.mean(its) > 0
