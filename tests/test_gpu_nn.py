"""The learned initial guess on the GPU: tensor-core kernels against the NumPy model, equivariance
of the features, and what a trained model gains over the untrained guess (mu4)."""

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
    """A 90-degree turn of a cubic box: invariants unchanged, vector channels and the graph field
    turned, for a first geometry and a displaced second one (the field-change channel nonzero)."""
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.learned import features
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(4, 1.25, seed=4)
    st = MDSettings(precision="double", cutoff=0.6, ewald_beta=6.0, pme_grid=(32, 32, 32))
    ff = PGMForceField(s, H, st)
    rng = np.random.default_rng(2)
    hist = rng.normal(scale=0.01, size=(4, s.n, 3))
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    dx = rng.normal(scale=2e-3, size=pos.shape)
    Hd = _dev(H[None], torch.float64)
    out = []
    for turn in (np.eye(3), R):
        p0 = _dev((pos @ turn.T) % 1.25, torch.float64)
        p1 = _dev(((pos + dx) @ turn.T) % 1.25, torch.float64)
        hd = _dev(hist @ turn.T, torch.float64)
        _, _, bl0 = features(ff, p0, Hd, hd)
        inv, vec, bl1 = features(ff, p1, Hd, hd, bl0)
        out.append((bl0.cpu().numpy()[:, :3], inv.cpu().numpy(), vec.cpu().numpy()))
    (b0, inv0, v0), (b1, inv1, v1) = out
    assert np.abs(b0 @ R.T - b1).max() <= 1e-5 * np.abs(b0).max()
    assert np.abs(v0[:, 0]).max() > 1e-3 * np.abs(v0[:, 1]).max()  # the field changed
    assert np.abs(inv0 - inv1).max() <= 1e-3 * max(1.0, np.abs(inv0).max())
    assert np.abs(v0 @ R.T - v1).max() <= 1e-4 * np.abs(v0).max()


def _same_positions(md, steps, ffs, captured=False):
    """Run `steps` MD steps of md (the learned guess; launched directly, or replayed from a captured
    graph) and solve every other force field in `ffs` (each with its own solver state, started from
    md's) at the same positions: per step CG iterations of md and of each of ffs."""
    import torch

    md.stream.synchronize()
    states = {k: md.ind.clone() for k in ffs}
    its = {"md": []}
    its.update({k: [] for k in ffs})
    if captured:
        md.capture()
    for _ in range(steps):
        if captured:
            md.run(1)
        else:
            md.step()
        md.stream.synchronize()
        its["md"].append(int(md.result.iterations[0]))
        assert float(md.result.residual[0]) <= md.ff.s.dipole_tol and not int(md.result.status[0]) & 0x2
        pos = md.pos.clone()
        for k, ff in ffs.items():
            r = ff.compute(pos, md.box[0].cpu().numpy(), None, states[k])
            states[k] = r.induction
            its[k].append(int(r.iterations[0]))
        torch.cuda.synchronize()
    return {k: np.array(v) for k, v in its.items()}


def _learned_md(prec="mixed", tol=1e-6):
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(5, 1.55, seed=6)
    kw = dict(precision=prec, cutoff=0.7, ewald_beta=5.0, pme_grid=(32, 32, 32), dipole_tol=tol, max_iter=100)
    ff = PGMForceField(s, H, MDSettings(predictor="nn", **kw))
    md = RigidMD(ff, pos, H, temperature=300.0, dt_fs=1.0, gamma_ps=5.0, seed=2)
    others = {p: PGMForceField(s, H, MDSettings(predictor=p, **kw)) for p in ("mu4", "mu1")}
    return s, H, ff, md, others


def test_trained_guess_saves_iterations_over_mu4_and_mu1():
    """Plain-solver MD writes (features, mu* - mu4 guess); GPU Adam steps train the model; on later
    frames mu4 + its correction is closer to mu* than mu4 (and mu4 than the previous step's
    dipoles), and on held-out MD with the model the solver needs fewer CG iterations than plain CG
    from mu4 and from the previous step's dipoles, solved at the same positions from the same
    history, all to the same tolerance."""
    from pgm_jax_b200.learned import GuessModel, collect, guess_errors

    s, H, ff, md, others = _learned_md()
    train = collect(md, 64)
    held = collect(md, 16)
    model = GuessModel(seed=0)
    before = guess_errors(model, held)
    model.train(train, iters=2000, batch=8192, lr=2e-3)
    after = guess_errors(model, held)
    print("guess rms", before, after)
    assert before["model"] == before["mu4"]  # the untrained model adds nothing
    assert before["mu4"] < before["mu1"]
    assert after["model"] < 0.9 * before["mu4"], (before, after)  # the trained model gains on unseen frames
    model.install(ff)
    its = _same_positions(md, 40, others, captured=True)
    print("iterations per step", {k: float(v.mean()) for k, v in its.items()})
    assert its["md"].mean() < its["mu4"].mean() < its["mu1"].mean(), {k: float(v.mean()) for k, v in its.items()}
    assert int(ff.nn_fallback_stats()["fallbacks"][0]) <= 4  # the trained model is rarely worse than mu4


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_bad_model_falls_back_to_mu4(prec):
    """A model with random output weights (its corrections several times the mu4 guess's error):
    every solve's start residual is above twice the record of mu4's, so every step falls back to
    x4 with one extra operator sweep, and needs at most one CG iteration more than mu4 at the same
    positions from the same history; the solution meets the tolerance."""
    from pgm_jax_b200.learned import N_HID, N_OUT, GuessModel, init_weights

    s, H, ff, md, others = _learned_md(prec, tol=1e-7)
    for _ in range(12):  # plain mu4 starts (no model yet) record the extrapolation's start residual
        md.step()
    md.stream.synchronize()
    assert ff.nn_fallback_stats()["ref_err"][0] > 0
    w = init_weights(0)
    rng = np.random.default_rng(9)
    w[-(N_HID * N_OUT + N_OUT):] = rng.normal(scale=0.5, size=N_HID * N_OUT + N_OUT)  # output layer
    GuessModel(w).install(ff)
    its = _same_positions(md, 3, {"mu4": others["mu4"]})  # host-driven solves
    its2 = _same_positions(md, 3, {"mu4": others["mu4"]}, captured=True)  # the fallback as a conditional node
    st = ff.nn_fallback_stats()
    assert int(st["fallbacks"][0]) == 6, st
    assert np.all(its["md"] <= its["mu4"] + 1) and np.all(its2["md"] <= its2["mu4"] + 1), (its, its2)
    ff.set_nn_fallback(0.0)  # without the check the bad guess costs iterations
    its_off = _same_positions(md, 4, {"mu4": others["mu4"]}, captured=True)
    assert its_off["md"].mean() > its_off["mu4"].mean() + 1, its_off
