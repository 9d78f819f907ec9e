"""The message-passing model of the learned guess on the GPU (csrc/pgm_mpnn.cu): its forward pass
and the gradient of its training loss against the NumPy restatement (oracle/nn_oracle.py, BF16
rounding at the same points, and the exact float64 gradient), and what the trained model gains
in MD over plain CG from mu4 and from the previous step's dipoles."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

import nn_oracle as N  # noqa: E402


def _graph(n, deg, rng, emax=128):
    """A random symmetric graph in the row build's edge format: per atom up to emax float4
    (x, y, z, partner bits), lengths in [0.1, 0.5) nm."""
    pairs = set()
    for i in range(n):
        for j in rng.choice(n, deg, replace=False):
            if j != i:
                pairs.add((min(i, j), max(i, j)))
    edges = np.zeros((n, emax, 4), np.float32)
    counts = np.zeros(n, np.int32)
    src, dst, dist = [], [], []
    for i, j in sorted(pairs):
        u = rng.normal(size=3)
        x = (u / np.linalg.norm(u) * rng.uniform(0.1, 0.5)).astype(np.float32)
        for a, b, v in ((i, j, x), (j, i, -x)):
            t = counts[a]
            edges[a, t, :3] = v
            edges[a, t, 3] = np.array([b], np.int32).view(np.float32)[0]
            counts[a] += 1
            src.append(a)
            dst.append(b)
            dist.append(float(np.sqrt(np.float32(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))))
    assert counts.max() <= emax
    return edges, counts, np.array(src), np.array(dst), np.array(dist)


def test_mpnn_forward_and_gradient_match_numpy():
    from pgm_jax_b200.learned import GRAPH_CUTOFF, SIGMA, MPNNModel

    rng = np.random.default_rng(2)
    n = 300  # not a multiple of the 128-row tile
    edges, counts, src, dst, dist = _graph(n, 12, rng)
    phi = N.radial(dist, GRAPH_CUTOFF)
    w = (rng.normal(scale=0.15, size=N.mpnn_nparam())).astype(np.float32)
    inv = rng.normal(size=(n, N.N_IN)).astype(np.float32)
    vec = rng.normal(scale=0.02, size=(n, N.N_CH, 3)).astype(np.float32)
    tgt = rng.normal(scale=2e-4, size=(n, 3)).astype(np.float32)
    dev = torch.device("cuda", 0)
    t = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    frame = {"inv": t(inv), "vec": t(vec), "target": t(tgt), "edges": t(edges), "counts": t(counts)}
    m = MPNNModel(w)
    mu = m.predict(frame).cpu().numpy()
    mu_ref, _ = N.mpnn_forward(w, inv, vec, src, dst, phi, SIGMA)
    assert np.abs(mu - mu_ref).max() <= 2e-3 * np.abs(mu_ref).max(), np.abs(mu - mu_ref).max() / np.abs(mu_ref).max()
    scale = 1.0 / (n * SIGMA**2)
    loss = m.loss_grad(frame, scale)
    g = m.g.cpu().numpy()
    loss_ref, g_ref = N.mpnn_loss_grad(w, inv, vec, src, dst, phi, tgt, SIGMA, scale)
    assert abs(loss - loss_ref) <= 2e-3 * loss_ref, (loss, loss_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-2 * np.linalg.norm(g_ref), np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    _, g_ex = N.mpnn_loss_grad(w, inv, vec, src, dst, phi, tgt, SIGMA, scale, rounded=False)
    assert np.linalg.norm(g - g_ex) <= 8e-2 * np.linalg.norm(g_ex)  # BF16 is the only approximation


def test_trained_mpnn_saves_iterations_over_mu4_and_mu1():
    """Plain-solver MD writes frames (features, graph, mu* - mu4 guess); GPU Adam steps on the
    project's forward and backward kernels train the message-passing model; on held-out frames its
    guess beats mu4, and on held-out MD the solver from it needs fewer CG iterations than plain CG
    from mu4 and from the previous step's dipoles (same positions, same history, same tolerance)."""
    from test_gpu_nn import _learned_md, _same_positions

    from pgm_jax_b200.learned import MPNNModel, collect_frames, frame_errors

    s, H, ff, md, others = _learned_md()
    train = collect_frames(md, 64)
    held = collect_frames(md, 16)
    model = MPNNModel(seed=0)
    before = frame_errors(model, held)
    model.train(train, iters=1500, lr=2e-3)
    after = frame_errors(model, held)
    print("guess rms", before, after)
    assert abs(before["model"] - before["mu4"]) <= 1e-9 * before["mu4"]  # the untrained model adds nothing
    assert after["model"] < 0.9 * before["mu4"], (before, after)
    model.install(ff)
    its = _same_positions(md, 40, others, captured=True)
    print("iterations per step", {k: float(v.mean()) for k, v in its.items()})
    assert its["md"].mean() < its["mu4"].mean() < its["mu1"].mean(), {k: float(v.mean()) for k, v in its.items()}
