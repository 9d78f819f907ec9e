"""NumPy restatement of the ring-polymer integrator pieces and the q-TIP4P/F water term -- TEST
INFRASTRUCTURE (only tests use it).

The free ring-polymer step in normal modes with the Cayley propagator, the PILE-L thermostat and
PILE-G's Bussi factor (pgm_jax/md/pimd.py:238-282, 411-440, 651-670; thermostats.py:279-335), and the q-TIP4P/F intramolecular energy
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


def free_step_centroid_scaled(q, p, C, omega, mass, dt, alpha):
    """A(dt/2), the centroid momentum times alpha (PILE-G's Bussi rescaling, no other friction),
    A(dt/2), in normal modes (pimd.py:411-440)."""
    qn = np.einsum("jl,jnc->lnc", C, q)
    pn = np.einsum("jl,jnc->lnc", C, p)
    w = np.asarray(omega)[:, None, None]
    m = np.asarray(mass)[None, :, None]
    qn, pn = cayley(qn, pn, w, m, 0.5 * dt)
    pn[0] *= alpha
    qn, pn = cayley(qn, pn, w, m, 0.5 * dt)
    return np.einsum("jl,lnc->jnc", C, qn), np.einsum("jl,lnc->jnc", C, pn)


def centroid_kinetic(p, C, mass):
    """Kinetic energy of the ring polymer's centroid mode: sum p~0^2 / (2 m), p~0 = sum_j C[j][0] p_j."""
    p0 = np.einsum("j,jnc->nc", C[:, 0], p)
    return float(0.5 * np.sum(p0 * p0 / np.asarray(mass)[:, None]))


def bussi_factor(K, kT, dof, h, tau, r1, S):
    """Bussi's rescaling factor for a step h given the draws R1 ~ N(0,1), S ~ chi^2(dof - 1)
    (thermostats.py:320-334)."""
    K = max(K, 1e-30)
    c = math.exp(-h / tau)
    f = 0.5 * dof * kT / (dof * K)
    a2 = c + (1.0 - c) * f * (r1 * r1 + S) + 2.0 * r1 * math.sqrt(c * (1.0 - c) * f)
    return math.copysign(math.sqrt(max(a2, 0.0)), r1 + math.sqrt(c / ((1.0 - c) * f)))


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
