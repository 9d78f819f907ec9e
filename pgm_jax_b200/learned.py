"""The learned initial guess of the induced-dipole solve: data, training and use.

A message-passing model on the short-range graph (edges r < 0.5 nm taken from the pair rows)
predicts the correction mu* - x4 from the mu4 extrapolation x4 = 4 mu1 - 6 mu2 + 4 mu3 - mu4 to the
converged induced dipoles mu* of a step, from the change of the graph's permanent field since the
last step (the real-space field of charges and permanent dipoles over the graph edges) and the last
steps' dipoles.  With predictor "nn" the engine's solver starts CG from x4 + the prediction with
mu4's fused start (one field sweep, as the reference's mu4 predictor) and iterates to the same
tolerance, so a poor guess costs iterations, never accuracy; the untrained (zero) model is mu4 exactly.
The model (csrc/pgm_nn.cu): 16 rotation invariants -> MLP 64 -> 64 (SiLU) -> 15 coefficients that
mix 15 vector channels per atom (csrc/pgm_kernels.cuh k_nn_chan, k_nn_features), so the prediction
rotates with the system.  Training runs on the GPU with the project's BF16 tensor-core
forward/backward kernels and Adam; the data are (features, mu* - x4) pairs written while the plain
solver runs MD.  The reference has no counterpart (pgm_jax/md/forcefield.py:1917-2008 has the mu3,
mu4 and least-squares predictors only).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

N_IN, N_HID, N_OUT, N_CH = 16, 64, 32, 15
SIGMA = 2e-4  # e nm, scale of the per-step changes in the invariants and the loss
GRAPH_CUTOFF = 0.5  # nm


def init_weights(seed: int = 0) -> np.ndarray:
    """Flat FP32 weights (w1, b1, w2, b2, w3, b3): small random hidden layers and a zero output
    layer, so the untrained model predicts no correction (the guess is mu4)."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(scale=1.0 / np.sqrt(N_IN), size=(N_IN, N_HID))
    w2 = rng.normal(scale=1.0 / np.sqrt(N_HID), size=(N_HID, N_HID))
    flat = np.concatenate([w1.ravel(), np.zeros(N_HID), w2.ravel(), np.zeros(N_HID), np.zeros(N_HID * N_OUT),
                           np.zeros(N_OUT)]).astype(np.float32)
    assert flat.size == _lib.load().pgm_nn_param_count()
    return flat


def _p(t: torch.Tensor):
    return C.c_void_p(t.data_ptr())


def features(ff, pos: torch.Tensor, boxes: torch.Tensor, hist: torch.Tensor, bl_prev: torch.Tensor | None = None):
    """Invariants (N, 16), vector channels (N, 15, 3) and the graph's permanent field (N, 4) at a
    geometry, with the history hist (4, N, 3) of the solve there.

    bl_prev: the previous step's graph field (else the field-change channel is zero).  Uses the
    installed sigma and graph cutoff (GuessModel.install) or the defaults."""
    n = ff.n
    inv = torch.empty((n, N_IN), dtype=torch.float32, device=ff.device)
    vec = torch.empty((n, N_CH, 3), dtype=torch.float32, device=ff.device)
    bl = torch.empty((n, 4), dtype=torch.float32, device=ff.device)
    _lib.check(ff._lib.pgm_nn_features(ff._h, ff._stream(), _p(pos), _p(boxes), _p(hist),
                                       None if bl_prev is None else _p(bl_prev), _p(bl), _p(inv), _p(vec)))
    return inv, vec, bl


class GuessModel:
    """Device weights of the model with its Adam state."""

    def __init__(self, weights: np.ndarray | None = None, device: int = 0, seed: int = 0) -> None:
        self.dev = torch.device("cuda", device)
        w = init_weights(seed) if weights is None else np.asarray(weights, np.float32)
        self.w = torch.tensor(w, device=self.dev)
        self.g = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.step = 0
        self.lib = _lib.load()

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def predict(self, inv: torch.Tensor, vec: torch.Tensor) -> torch.Tensor:
        mu = torch.empty((inv.shape[0], 3), dtype=torch.float32, device=self.dev)
        _lib.check(self.lib.pgm_nn_predict(self._stream(), _p(self.w), _p(inv), _p(vec), int(inv.shape[0]), _p(mu)))
        return mu

    def loss_grad(self, inv, vec, target, scale: float) -> float:
        """Adds d loss / d w to self.g; returns loss = scale * sum |mu - target|^2."""
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        _lib.check(self.lib.pgm_nn_loss_grad(self._stream(), _p(self.w), _p(inv), _p(vec), _p(target), int(inv.shape[0]),
                                             float(scale), _p(self.g), _p(loss)))
        return float(loss.item())

    def adam(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step += 1
        _lib.check(self.lib.pgm_nn_adam(self._stream(), _p(self.w), _p(self.g), _p(self.m), _p(self.v), lr, beta1, beta2, eps,
                                        self.step))

    def train(self, data: dict, iters: int = 400, batch: int = 16384, lr: float = 2e-3, seed: int = 0, log=None) -> list:
        """Adam on minibatches of (inv, vec, target) (dict of device tensors); returns the losses
        (mean |mu - target|^2 / SIGMA^2 per atom)."""
        n = data["inv"].shape[0]
        g = torch.Generator(device=self.dev)
        g.manual_seed(seed)
        losses = []
        for it in range(iters):
            idx = torch.randint(0, n, (min(batch, n),), device=self.dev, generator=g)
            scale = 1.0 / (idx.numel() * SIGMA**2)
            loss = self.loss_grad(data["inv"][idx].contiguous(), data["vec"][idx].contiguous(), data["target"][idx].contiguous(),
                                  scale)
            lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * it / iters))  # cosine decay
            self.adam(lr=lr_t)
            losses.append(loss)
            if log and (it % 100 == 0 or it == iters - 1):
                log(f"  train {it:5d}  loss {loss:.4e}")
        return losses

    def install(self, ff) -> None:
        """Use the model as the solver's initial guess (predictor "nn")."""
        _lib.check(ff._lib.pgm_set_nn_model(ff._h, _p(self.w), SIGMA, GRAPH_CUTOFF))


def collect(md, steps: int, every: int = 1) -> dict:
    """Run `steps` MD steps with the plain solver and keep, for every `every`-th step once the
    history holds four steps, the features and the target mu* - x4 (device tensors; "prev" holds
    mu1 - x4, for the previous-step guess's error)."""
    ff = md.ff
    keep = {"inv": [], "vec": [], "target": [], "prev": []}
    bl_prev = None
    for k in range(steps):
        md.stream.synchronize()
        count = int(md.ind.count.min())
        with torch.cuda.stream(md.stream):  # everything on the MD stream, in order
            hist = md.ind.hist.clone()
        md.step()
        with torch.cuda.stream(md.stream):
            inv, vec, bl = features(ff, md.pos, md.box, hist, bl_prev)
            x4 = 4.0 * hist[0] - 6.0 * hist[1] + 4.0 * hist[2] - hist[3]
            target = (md.ind.mu - x4).to(torch.float32)
            prev = (hist[0] - x4).to(torch.float32)
        md.stream.synchronize()
        if count >= 4 and bl_prev is not None and k % every == 0:
            keep["inv"].append(inv)
            keep["vec"].append(vec)
            keep["target"].append(target)
            keep["prev"].append(prev)
        bl_prev = bl
    return {k: torch.cat(v) for k, v in keep.items()}


def guess_errors(model: GuessModel, data: dict) -> dict:
    """RMS error (e nm) of the guesses on data: mu4 + the model's correction, mu4, and the previous
    step's dipoles."""
    pred = model.predict(data["inv"], data["vec"])
    t = data["target"]
    rms = lambda x: float(torch.sqrt(torch.mean(x * x)))  # noqa: E731
    return {"model": rms(pred - t), "mu4": rms(t), "mu1": rms(data["prev"] - t)}


# ----------------------------------------------------------------------------- message passing
EMAX = 128  # graph edges kept per atom (the row build's list)
# W0, b0, per layer (W_g, W_f, W_a, b_a, W_b, b_b), W_o, b_o: (out, in) matrices
MPNN_SHAPES = [(64, 16), (64,)] + [(16, 64), (16, 8), (64, 80), (64,), (64, 64), (64,)] * 2 + [(16, 64), (16,)]


def mpnn_init_weights(seed: int = 0) -> np.ndarray:
    """Flat FP32 weights of the message-passing model (csrc/pgm_mpnn.cu): random input, message,
    filter and update layers (the filters and the residual branches scaled down), a zero output
    layer, so the untrained model predicts no correction (the guess is mu4)."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, shape in enumerate(MPNN_SHAPES):
        role = (k - 2) % 6 if 2 <= k < 14 else None  # 0 W_g, 1 W_f, 2 W_a, 4 W_b
        if len(shape) == 1 or k == len(MPNN_SHAPES) - 2:  # biases, W_o
            parts.append(np.zeros(shape))
        else:
            scale = 1.0 / np.sqrt(shape[1]) * (0.3 if role in (1, 4) else 1.0)
            parts.append(rng.normal(scale=scale, size=shape))
    flat = np.concatenate([p.ravel() for p in parts]).astype(np.float32)
    assert flat.size == _lib.load().pgm_mpnn_param_count()
    return flat


class MPNNModel:
    """The 2-layer message-passing model of the learned guess on the short-range graph (device
    weights and Adam state): per atom an embedding of the 16 invariants, two rounds of messages
    along the graph's edges expanded in 8 radial functions, and the coefficients of the 15 vector
    channels (csrc/pgm_mpnn.cu; its dense layers on the tcgen05 tensor cores)."""

    def __init__(self, weights: np.ndarray | None = None, device: int = 0, seed: int = 0) -> None:
        self.dev = torch.device("cuda", device)
        w = mpnn_init_weights(seed) if weights is None else np.asarray(weights, np.float32)
        self.w = torch.tensor(w, device=self.dev)
        self.g = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.step = 0
        self.lib = _lib.load()
        self._work = {}

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.dev).cuda_stream)

    def _ws(self, n: int, train: bool) -> torch.Tensor:
        key = (n, train)
        if key not in self._work:
            self._work[key] = torch.empty(int(self.lib.pgm_mpnn_work_bytes(n, int(train))), dtype=torch.uint8, device=self.dev)
        return self._work[key]

    def predict(self, frame: dict) -> torch.Tensor:
        n = frame["inv"].shape[0]
        mu = torch.empty((n, 3), dtype=torch.float32, device=self.dev)
        _lib.check_mpnn(self.lib.pgm_mpnn_predict(self._stream(), _p(self.w), _p(frame["inv"]), _p(frame["vec"]),
                                                  _p(frame["edges"]), _p(frame["counts"]), EMAX, n, SIGMA, GRAPH_CUTOFF,
                                                  _p(self._ws(n, False)), _p(mu)))
        return mu

    def loss_grad(self, frame: dict, scale: float) -> float:
        """Adds d loss / d w to self.g; returns loss = scale * sum |mu - target|^2."""
        n = frame["inv"].shape[0]
        loss = torch.zeros(1, dtype=torch.float64, device=self.dev)
        _lib.check_mpnn(self.lib.pgm_mpnn_loss_grad(self._stream(), _p(self.w), _p(frame["inv"]), _p(frame["vec"]),
                                                    _p(frame["target"]), _p(frame["edges"]), _p(frame["counts"]), EMAX, n,
                                                    SIGMA, GRAPH_CUTOFF, float(scale), _p(self._ws(n, True)), _p(self.g),
                                                    _p(loss)))
        return float(loss.item())

    def adam(self, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.step += 1
        _lib.check_mpnn(self.lib.pgm_mpnn_adam(self._stream(), _p(self.w), _p(self.g), _p(self.m), _p(self.v), lr, beta1,
                                               beta2, eps, self.step))

    def train(self, frames: list, iters: int = 1000, lr: float = 2e-3, seed: int = 0, log=None) -> list:
        """Adam with one whole frame (its graph) per step, frames in a seeded random order; returns
        the losses (mean |mu - target|^2 / SIGMA^2 per atom)."""
        rng = np.random.default_rng(seed)
        losses = []
        for it in range(iters):
            f = frames[int(rng.integers(len(frames)))]
            scale = 1.0 / (f["inv"].shape[0] * SIGMA**2)
            loss = self.loss_grad(f, scale)
            self.adam(lr=lr * 0.5 * (1.0 + np.cos(np.pi * it / iters)))
            losses.append(loss)
            if log and (it % 100 == 0 or it == iters - 1):
                log(f"  train {it:5d}  loss {loss:.4e}")
        return losses

    def install(self, ff) -> None:
        """Use the model as the solver's initial guess (predictor "nn")."""
        _lib.check(ff._lib.pgm_set_mpnn_model(ff._h, _p(self.w), SIGMA, GRAPH_CUTOFF))


def collect_frames(md, steps: int) -> list:
    """As collect(), frame by frame with each frame's graph (edges (N, EMAX, 4) float32 as the row
    build writes them, counts (N,) int32): the training data of the message-passing model."""
    ff = md.ff
    frames = []
    bl_prev = None
    for _ in range(steps):
        md.stream.synchronize()
        count = int(md.ind.count.min())
        with torch.cuda.stream(md.stream):
            hist = md.ind.hist.clone()
        md.step()
        with torch.cuda.stream(md.stream):
            inv, vec, bl = features(ff, md.pos, md.box, hist, bl_prev)
            x4 = 4.0 * hist[0] - 6.0 * hist[1] + 4.0 * hist[2] - hist[3]
            target = (md.ind.mu - x4).to(torch.float32)
            prev = (hist[0] - x4).to(torch.float32)
            edges = torch.empty((ff.n, EMAX, 4), dtype=torch.float32, device=ff.device)
            counts = torch.empty(ff.n, dtype=torch.int32, device=ff.device)
            _lib.check(ff._lib.pgm_nn_graph(ff._h, ff._stream(), _p(edges), _p(counts), EMAX))
        md.stream.synchronize()
        if count >= 4 and bl_prev is not None:
            frames.append({"inv": inv, "vec": vec, "target": target, "prev": prev, "edges": edges, "counts": counts})
        bl_prev = bl
    return frames


def frame_errors(model: MPNNModel, frames: list) -> dict:
    """RMS error (e nm) over frames of mu4 + the model's correction, mu4 and the previous step's dipoles."""
    se = {"model": 0.0, "mu4": 0.0, "mu1": 0.0}
    cnt = 0
    for f in frames:
        pred = model.predict(f)
        t = f["target"]
        se["model"] += float(torch.sum((pred - t) ** 2))
        se["mu4"] += float(torch.sum(t * t))
        se["mu1"] += float(torch.sum((f["prev"] - t) ** 2))
        cnt += t.numel()
    return {k: float(np.sqrt(v / cnt)) for k, v in se.items()}


def random_frame(n: int, degree: int = 52, seed: int = 0, device: int = 0) -> dict:
    """A seeded synthetic frame of the message-passing model's inputs on the device: n atoms with
    `degree` edges each (random partners, lengths uniform in [0.1, 0.5) nm, random directions), the
    16 invariants N(0, 1) and the 15 vector channels N(0, 0.02^2) -- the sizes of a water box's
    0.5 nm graph (about 52 edges per atom), for timing and profiling the inference kernels."""
    dev = torch.device("cuda", device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    edges = torch.zeros((n, EMAX, 4), device=dev)
    d = torch.randn((n, degree, 3), device=dev, generator=g)
    d = d / d.norm(dim=-1, keepdim=True) * (0.1 + 0.4 * torch.rand((n, degree, 1), device=dev, generator=g))
    edges[:, :degree, :3] = d
    edges[:, :degree, 3] = torch.randint(0, n, (n, degree), device=dev, generator=g, dtype=torch.int32).view(torch.float32)
    return {"inv": torch.randn((n, N_IN), device=dev, generator=g),
            "vec": 0.02 * torch.randn((n, N_CH, 3), device=dev, generator=g),
            "edges": edges, "counts": torch.full((n,), degree, dtype=torch.int32, device=dev),
            "target": 1e-4 * torch.randn((n, 3), device=dev, generator=g)}


def _time_inference(n: int, reps: int = 20) -> None:
    """Mean time of the message-passing model's inference (pgm_mpnn_predict: weight conversion and
    the five kernels) on a synthetic frame of n atoms, CUDA events on the current stream."""
    frame = random_frame(n)
    m = MPNNModel()
    for _ in range(3):
        m.predict(frame)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        m.predict(frame)
    b.record()
    torch.cuda.synchronize()
    print(f"message-passing inference, {n} atoms: {a.elapsed_time(b) / reps * 1e3:.1f} us per call")


if __name__ == "__main__":
    import sys

    _time_inference(int(sys.argv[1]) if len(sys.argv) > 1 else 98304)
