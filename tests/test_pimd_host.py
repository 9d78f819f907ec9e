"""Ring-polymer pieces on the host: the normal modes and frequencies (pgm_jax/md/pimd.py:135-236),
the mode frictions of PILE / TRPMD / RPMD, and the oracle's free step (energy of every free mode
conserved, orthonormal transforms)."""

import math

import numpy as np
import pytest

import pimd_oracle as PO
from pgm_jax_b200.pimd import HBAR, KB, RingPolymer, frictions, normal_modes


@pytest.mark.parametrize("P", [1, 2, 5, 8, 32])
def test_normal_modes_orthonormal_and_ordered(P):
    C, idx = normal_modes(P)
    assert np.allclose(C.T @ C, np.eye(P), atol=1e-13) and np.allclose(C @ C.T, np.eye(P), atol=1e-13)
    assert np.all(np.diff(idx) >= 0) and idx[0] == 0
    assert np.allclose(C[:, 0], 1 / math.sqrt(P))
    if P % 2 == 0 and P > 1:
        assert np.allclose(C[:, -1], (-1.0) ** np.arange(P) / math.sqrt(P))
    ring = RingPolymer(P, 300.0)
    assert np.isclose(ring.omega_P, P * KB * 300.0 / HBAR)
    assert np.allclose(ring.omega, 2 * ring.omega_P * np.sin(np.pi * idx / P))
    # the spring energy is the normal-mode sum of m omega_l^2 |q~_l|^2 / 2
    rng = np.random.default_rng(P)
    q = rng.normal(size=(P, 4, 3))
    m = rng.uniform(1, 16, size=4)
    qn = np.einsum("jl,jnc->lnc", C, q)
    modes = 0.5 * m * np.sum(ring.omega[:, None, None] ** 2 * qn**2, axis=(0, 2))
    assert np.allclose(ring.spring(q, m), modes, rtol=1e-10)


def test_frictions():
    ring = RingPolymer(8, 300.0)
    g = frictions(ring, "pimd", 0.2)
    assert np.isclose(g[0], 5.0) and np.allclose(g[1:], 2 * ring.omega[1:])
    assert frictions(ring, "trpmd")[0] == 0 and np.allclose(frictions(ring, "trpmd")[1:], ring.omega[1:])
    assert np.all(frictions(ring, "rpmd") == 0)
    with pytest.raises(ValueError):
        frictions(ring, "nve")
    g = frictions(ring, "pimd", 0.2, centroid="g")  # PILE-G: the centroid is Bussi's, not Langevin's
    assert g[0] == 0 and np.allclose(g[1:], 2 * ring.omega[1:])
    with pytest.raises(ValueError):
        frictions(ring, "pimd", centroid="x")


def test_bussi_factor_keeps_the_canonical_kinetic_energy():
    """With exact draws, K alpha^2 has mean c K + (1 - c) K0 (Bussi's relaxation toward K0 = N_f kT / 2)."""
    import pimd_oracle as PO

    rng = np.random.default_rng(0)
    dof, kT, h, tau, K = 300.0, 2.5, 0.0005, 0.2, 500.0
    K0 = 0.5 * dof * kT
    a = np.array([PO.bussi_factor(K, kT, dof, h, tau, rng.normal(), rng.chisquare(dof - 1)) for _ in range(100000)])
    c = np.exp(-h / tau)
    mean = np.mean(K * a * a)
    assert abs(mean - (c * K + (1 - c) * K0)) < 4 * np.std(K * a * a) / np.sqrt(len(a))
    assert np.all(a > 0)  # far from K = 0 the factor keeps its sign


def test_oracle_free_step_conserves_every_mode():
    P, n = 8, 5
    ring = RingPolymer(P, 300.0)
    rng = np.random.default_rng(0)
    q, p = rng.normal(scale=0.01, size=(P, n, 3)), rng.normal(size=(P, n, 3))
    m = rng.uniform(1, 16, size=n)

    def mode_energy(q, p):
        qn = np.einsum("jl,jnc->lnc", ring.C, q)
        pn = np.einsum("jl,jnc->lnc", ring.C, p)
        return np.sum(pn**2 / (2 * m[None, :, None]), axis=(1, 2)) + 0.5 * np.sum(
            m[None, :, None] * ring.omega[:, None, None] ** 2 * qn**2, axis=(1, 2))

    e0 = mode_energy(q, p)
    for _ in range(20):
        q, p = PO.free_step(q, p, ring.C, ring.omega, m, 0.0005)
    assert np.allclose(mode_energy(q, p), e0, rtol=1e-12)
