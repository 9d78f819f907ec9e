"""NumPy restatement of the ring-polymer integrator pieces and the q-TIP4P/F water term -- TEST
INFRASTRUCTURE (only tests use it).

The free ring-polymer step in normal modes with the Cayley propagator and the PILE-L thermostat
(pgm_jax/md/pimd.py:238-282, 411-440, 651-670), and the q-TIP4P/F intramolecular energy
(pgm_jax/models/water.py:38-69) with forces by central differences.
"""

from __future__ import annotations

import math

import numpy as np


def cayley(q, p, w, m, h):
    """One Cayley step of length h: p' = [(1 - x) p - m w^2 h q] / (1 + x), q' = [h p / m + (1 - x) q] / (1 + x),
    x = (w h / 2)^2 (w per mode (P, 1, 1), m per atom (1, N, 1))."""
    x = 0.25 * (w * h) ** 2
    den = 1.0 + x
    pn = ((1.0 - x) * p - m * w * w * h * q) / den
    qn = (h * p / m + (1.0 - x) * q) / den
    return qn, pn


def free_step(q, p, C, omega, mass, dt):
    """A(dt/2) O(none) A(dt/2) in normal modes on bead arrays q, p (P, N, 3): the deterministic part
    of the integrator's middle (with zero friction it is the whole A O A)."""
    qn = np.einsum("jl,jnc->lnc", C, q)
    pn = np.einsum("jl,jnc->lnc", C, p)
    w = np.asarray(omega)[:, None, None]
    m = np.asarray(mass)[None, :, None]
    qn, pn = cayley(qn, pn, w, m, 0.5 * dt)
    qn, pn = cayley(qn, pn, w, m, 0.5 * dt)
    return np.einsum("jl,lnc->jnc", C, qn), np.einsum("jl,lnc->jnc", C, pn)


def qtip4pf_energy(R, D, alpha, r_eq, k_theta, theta_eq_rad):
    """q-TIP4P/F energy of one water R (3, 3) = O, H, H [nm]."""
    u, v = R[1] - R[0], R[2] - R[0]
    r1, r2 = np.linalg.norm(u), np.linalg.norm(v)
    th = math.acos(max(-1.0, min(1.0, float(u @ v) / (r1 * r2))))

    def morse4(r):
        x = alpha * (r - r_eq)
        return D * (x * x - x**3 + 7.0 / 12.0 * x**4)

    return morse4(r1) + morse4(r2) + 0.5 * k_theta * (th - theta_eq_rad) ** 2


def qtip4pf_forces(R, prm, h=1e-6):
    """(energy, forces (3, 3)) of one water by central differences."""
    F = np.zeros((3, 3))
    for a in range(3):
        for c in range(3):
            Rp, Rm = R.copy(), R.copy()
            Rp[a, c] += h
            Rm[a, c] -= h
            F[a, c] = -(qtip4pf_energy(Rp, *prm) - qtip4pf_energy(Rm, *prm)) / (2 * h)
    return qtip4pf_energy(R, *prm), F
