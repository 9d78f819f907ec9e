"""NumPy restatement of the learned-guess model and its gradient -- TEST INFRASTRUCTURE.

The same MLP as pgm_jax_b200/csrc/pgm_nn.cu (16 invariants -> 64 -> 64 SiLU -> 32 coefficients,
mu = sum_c c_c v_c over 15 vector channels), with the BF16 roundings at the points where the
tensor-core kernels round (inputs, weights, hidden activations, backpropagated errors), in float64
otherwise; and the exact float64 model for finite-difference checks.  Only tests use it.
"""

from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT, N_CH = 16, 64, 32, 15


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(flat: np.ndarray):
    o = 0
    out = []
    for shape in ((N_IN, N_HID), (N_HID,), (N_HID, N_HID), (N_HID,), (N_HID, N_OUT), (N_OUT,)):
        size = int(np.prod(shape))
        out.append(np.asarray(flat[o:o + size], np.float64).reshape(shape))
        o += size
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(flat, inv, vec, rounded: bool = True):
    r = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(flat)
    x = r(inv)
    z1 = x @ r(w1) + b1
    a1 = r(silu(z1))
    z2 = a1 @ r(w2) + b2
    a2 = r(silu(z2))
    c = a2 @ r(w3) + b3
    mu = np.einsum("nc,nca->na", c[:, :N_CH], np.asarray(vec, np.float64))
    return mu, (x, z1, a1, z2, a2, c)


def loss_grad(flat, inv, vec, target, scale: float, rounded: bool = True):
    """(loss, flat gradient) of scale * sum |mu - target|^2, rounded like the GPU kernels."""
    r = bf16 if rounded else (lambda a: np.asarray(a, np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(flat)
    mu, (x, z1, a1, z2, a2, c) = forward(flat, inv, vec, rounded)
    e = mu - np.asarray(target, np.float64)
    loss = scale * np.sum(e * e)
    gc = np.zeros_like(c)
    gc[:, :N_CH] = 2.0 * scale * np.einsum("na,nca->nc", e, np.asarray(vec, np.float64))
    dz3 = r(gc)
    gw3 = a2.T @ dz3
    gb3 = gc.sum(0)
    dz2 = (dz3 @ r(w3).T) * dsilu(z2)
    gb2 = dz2.sum(0)
    dz2r = r(dz2)
    gw2 = a1.T @ dz2r
    dz1 = (dz2r @ r(w2).T) * dsilu(z1)
    gb1 = dz1.sum(0)
    gw1 = x.T @ r(dz1)
    return loss, np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3.ravel(), gb3])
