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


# ----------------------------------------------------------------------------- message passing
# The 2-layer message-passing model of csrc/pgm_mpnn.cu: per atom h0 = SiLU(W0 inv + b0) (64);
# per layer g = W_g h (16 message features) and a continuous-filter convolution over the graph's
# edges (Schuett et al., SchNet, 2017): s_i[r, f] = sum over edges (i, j) of phi_r(d_ij) g_j[f],
# a_i[f] = sum_r W_f[f, r] s_i[r, f] (the filter psi_f(d) = sum_r W_f[f, r] phi_r(d) is linear in
# the 8 radial functions); u = SiLU(W_a [h; a] + b_a) (80 -> 64), h <- h + W_b u + b_b;
# coefficients c = W_o h + b_o (16, the first 15 used) and the prediction SIGMA sum_c c_c v_c.
# Weight matrices are (out, in); BF16 rounding where the tensor-core path rounds (GEMM operands,
# h, g, a, u, and the radial values of the forward sums), FP32-like sums elsewhere (here float64).
M_HID, M_R, M_F, M_COEF = 64, 8, 16, 16
MPNN_SHAPES = [(64, 16), (64,)] + [(M_F, 64), (M_F, M_R), (64, 64 + M_F), (64,), (64, 64), (64,)] * 2 + [(16, 64), (16,)]
_PER_LAYER = 6


def mpnn_nparam() -> int:
    return int(sum(np.prod(s) for s in MPNN_SHAPES))


def mpnn_unpack(flat):
    """(W0, b0, [(Wg, Wf, Wa, ba, Wb, bb)] * 2, Wo, bo) in float64."""
    o, out = 0, []
    for shape in MPNN_SHAPES:
        size = int(np.prod(shape))
        out.append(np.asarray(flat[o:o + size], np.float64).reshape(shape))
        o += size
    W0, b0 = out[0], out[1]
    layers = [out[2 + _PER_LAYER * l: 2 + _PER_LAYER * (l + 1)] for l in range(2)]
    return W0, b0, layers, out[-2], out[-1]


def radial(d, rg):
    """phi_r(d), r = 0..7: Gaussians at r rg / 7 of width rg / 7 times the cosine cutoff, (E, 8) float32."""
    d = np.asarray(d, np.float32)[:, None]
    mu = np.arange(M_R, dtype=np.float32)[None, :] * np.float32(rg / (M_R - 1))
    gam = np.float32(((M_R - 1) / rg) ** 2)
    fc = np.float32(0.5) * (np.cos(np.float32(np.pi) * d / np.float32(rg)) + np.float32(1))
    return (np.exp(-gam * (d - mu) ** 2) * fc).astype(np.float64)


def _sums(g, src, dst, phi):
    """s[i, r, f] = sum over edges e with src[e] = i of phi[e, r] g[dst[e], f]."""
    n = g.shape[0]
    msg = np.einsum("er,ef->erf", phi, g[dst])
    s = np.zeros((n, M_R, M_F))
    np.add.at(s, src, msg)
    return s


def _sums_t(da, Wf, src, dst, phi, n):
    """The transposed convolution: dg[j, f] = sum over edges e with dst[e] = j of
    sum_r phi[e, r] W_f[f, r] da[src[e], f]."""
    contrib = (phi @ Wf.T) * da[src]
    dg = np.zeros((n, M_F))
    np.add.at(dg, dst, contrib)
    return dg


def mpnn_forward(flat, inv, vec, src, dst, phi, sigma, rounded=True):
    """Prediction (n, 3) and the cache of the backward pass."""
    r = bf16 if rounded else (lambda x: np.asarray(x, np.float64))
    W0, b0, layers, Wo, bo = mpnn_unpack(flat)
    x0 = r(inv)
    z0 = x0 @ r(W0).T + b0
    h = r(silu(z0))
    cache = {"x0": x0, "z0": z0, "layers": []}
    for Wg, Wf, Wa, ba, Wb, bb in layers:
        g = r(h @ r(Wg).T)
        s = _sums(g, src, dst, r(phi))  # the forward sums take the radial values in BF16 (tensor-core operands)
        a = r(np.einsum("nrf,fr->nf", s, Wf))
        Z = np.concatenate([h, a], 1)
        zu = Z @ r(Wa).T + ba
        u = r(silu(zu))
        hn = r(h + (u @ r(Wb).T + bb))
        cache["layers"].append({"h": h, "g": g, "s": s, "Z": Z, "zu": zu, "u": u})
        h = hn
    c = h @ r(Wo).T + bo
    cache["h2"] = h
    cache["c"] = c
    mu = sigma * np.einsum("nc,nck->nk", c[:, :N_CH], vec)
    return mu, cache


def mpnn_loss_grad(flat, inv, vec, src, dst, phi, target, sigma, scale, rounded=True):
    """loss = scale sum |mu - target|^2 and its gradient with respect to the flat weights."""
    r = bf16 if rounded else (lambda x: np.asarray(x, np.float64))
    W0, b0, layers, Wo, bo = mpnn_unpack(flat)
    n = inv.shape[0]
    mu, C = mpnn_forward(flat, inv, vec, src, dst, phi, sigma, rounded)
    e = mu - target
    loss = scale * np.sum(e * e)
    dmu = 2.0 * scale * e
    dc = np.zeros((n, M_COEF))
    dc[:, :N_CH] = sigma * np.einsum("nk,nck->nc", dmu, vec)
    gWo = dc.T @ C["h2"]
    gbo = dc.sum(0)
    dh = r(dc) @ r(Wo)
    lg = []
    for (Wg, Wf, Wa, ba, Wb, bb), L in zip(layers[::-1], C["layers"][::-1]):
        gWb = dh.T @ L["u"]
        gbb = dh.sum(0)
        du = r(dh) @ r(Wb)
        dzu = du * dsilu(L["zu"])
        gWa = dzu.T @ L["Z"]
        gba = dzu.sum(0)
        dZ = r(dzu) @ r(Wa)
        da = dZ[:, 64:]
        gWf = np.einsum("nf,nrf->fr", da, L["s"])
        dg = _sums_t(da, Wf, src, dst, phi, n)
        gWg = dg.T @ L["h"]
        dh = dh + dZ[:, :64] + r(dg) @ r(Wg)
        lg.append((gWg, gWf, gWa, gba, gWb, gbb))
    dz0 = dh * dsilu(C["z0"])
    gW0 = dz0.T @ C["x0"]
    gb0 = dz0.sum(0)
    flat_g = [gW0.ravel(), gb0]
    for t in lg[::-1]:
        flat_g += [x.ravel() for x in t]
    flat_g += [gWo.ravel(), gbo]
    return loss, np.concatenate(flat_g)
