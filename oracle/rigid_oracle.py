"""NumPy restatement of the reference's rigid-molecule NVE step -- TEST INFRASTRUCTURE, NOT THE PRODUCT.

pGM-JAX integrates rigid molecules with JAX-MD's rigid bodies (centre of mass + unit quaternion,
pgm_jax/md/rigid.py:94-304) and NO_SQUISH free-rotor splitting (pgm_jax/md/integrate.py:743-761
calls jax_md.simulate.momentum_step / position_step; jax-md >= 0.2.29 is a dependency that is not
vendored in the reference).  This file restates the published algorithm of Miller, Eleftheriou,
Pattnaik, Ndirango, Newns and Martyna, J. Chem. Phys. 116, 8649 (2002) ("NO_SQUISH"), with the body
set-up of rigid.py, so that the 10-step NVE install check of the reference (tests/test_water512.py)
can be reproduced on the CPU with the FP64 oracle's forces, and the GPU integrator compared with it.

Conventions (rigid.py and the paper):
  * quaternion q = (q0, q1, q2, q3), body -> space, rotate(q, s) = q s q*; the permutations
    P1 q = q (x) i = (-q1, q0, q3, -q2), P2 q = q (x) j = (-q2, -q3, q0, q1),
    P3 q = q (x) k = (-q3, q2, -q1, q0);
  * conjugate momentum p = 2 q (x) (0, L) with L the body-frame angular momentum, so
    L_k = (P_k q) . p / 2; the quaternion force of a body torque t is 2 q (x) (0, t);
  * free rotation about principal axis k for a time h: zeta = h (p . P_k q) / (4 I_k),
    q <- cos(zeta) q + sin(zeta) P_k q, p <- cos(zeta) p + sin(zeta) P_k p;
  * the free rotor for a time h: axis 3 for h/2, axis 2 for h/2, axis 1 for h, axis 2 for h/2,
    axis 3 for h/2 (principal moments ascending, I1 <= I2 <= I3);
  * NVE velocity Verlet (integrate.py:743-761): p += F dt/2; R += dt P/M and the free rotor for dt;
    forces; p += F dt/2.
Units: nm, ps, amu, kJ/mol.
"""

from __future__ import annotations

import numpy as np

KB = 0.0083144626181532  # kJ/mol/K (pgm_jax/units.py:16)


def quat_mul(a, b):
    """Hamilton product of quaternion arrays (..., 4)."""
    a0, a1, a2, a3 = np.moveaxis(a, -1, 0)
    b0, b1, b2, b3 = np.moveaxis(b, -1, 0)
    return np.stack([a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3, a0 * b1 + a1 * b0 + a2 * b3 - a3 * b2,
                     a0 * b2 - a1 * b3 + a2 * b0 + a3 * b1, a0 * b3 + a1 * b2 - a2 * b1 + a3 * b0], -1)


def perm(k: int, q):
    """P_k q = q (x) e_k (k = 1, 2, 3)."""
    q0, q1, q2, q3 = np.moveaxis(q, -1, 0)
    if k == 1:
        return np.stack([-q1, q0, q3, -q2], -1)
    if k == 2:
        return np.stack([-q2, -q3, q0, q1], -1)
    return np.stack([-q3, q2, -q1, q0], -1)


def rotation_matrix(q):
    """(M, 3, 3) body -> space rotation of unit quaternions (M, 4)."""
    w, x, y, z = np.moveaxis(q, -1, 0)
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def matrix_to_quaternion(R):
    """Unit quaternion with w >= 0 of a rotation matrix (Shepperd's branch on the largest element)."""
    R = np.asarray(R, float)
    t = np.trace(R)
    if t > 0:
        s = 2.0 * np.sqrt(t + 1.0)
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = 2.0 * np.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2])
        q = [(R[2, 1] - R[1, 2]) / s, 0.25 * s, (R[0, 1] + R[1, 0]) / s, (R[0, 2] + R[2, 0]) / s]
    elif R[1, 1] > R[2, 2]:
        s = 2.0 * np.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2])
        q = [(R[0, 2] - R[2, 0]) / s, (R[0, 1] + R[1, 0]) / s, 0.25 * s, (R[1, 2] + R[2, 1]) / s]
    else:
        s = 2.0 * np.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1])
        q = [(R[1, 0] - R[0, 1]) / s, (R[0, 2] + R[2, 0]) / s, (R[1, 2] + R[2, 1]) / s, 0.25 * s]
    q = np.array(q)
    return q / np.linalg.norm(q) * (1 if q[0] >= 0 else -1)


class RigidNVE:
    """Rigid molecules of one system (all instances of a Molecule object share the first one's
    principal frame, rigid.py:126-205), NVE velocity Verlet with the NO_SQUISH free rotor.

    force_fn(pos (N, 3)) -> (forces (N, 3), potential energy) is called once per step.
    """

    def __init__(self, system, pos, H, vel, force_fn) -> None:
        pos, H = np.asarray(pos, float), np.asarray(H, float)
        self.sys, self.H, self.force_fn = system, H, force_fn
        m = np.asarray(system.masses, float)
        Hinv = np.linalg.inv(H)
        templates = {}
        M = system.nmol
        self.local = np.zeros((system.n, 3))
        self.mass = np.zeros(M)
        self.I = np.zeros((M, 3))
        self.R = np.zeros((M, 3))
        self.q = np.zeros((M, 4))
        for k, mol in enumerate(system.molecules):
            a0, a1 = system.mol_start[k], system.mol_start[k + 1]
            x = pos[a0:a1]
            d = x - x[0]
            for _ in range(2):  # whole molecule: every atom at the minimum image of the first
                d = d - np.round(d @ Hinv) @ H
            x = x[0] + d
            mk = m[a0:a1]
            com = (mk[:, None] * x).sum(0) / mk.sum()
            y = x - com
            if id(mol) not in templates:
                It = (mk[:, None, None] * (np.sum(y * y, 1)[:, None, None] * np.eye(3) - y[:, :, None] * y[:, None, :])).sum(0)
                ev, U = np.linalg.eigh(It)
                if np.linalg.det(U) < 0:
                    U[:, 0] = -U[:, 0]
                templates[id(mol)] = (y @ U, ev)
            body, ev = templates[id(mol)]
            A = body.T @ y  # Kabsch: y ~ body @ Rk.T
            U_, _, Vt = np.linalg.svd(A)
            dd = np.sign(np.linalg.det(Vt.T @ U_.T))
            Rk = Vt.T @ np.diag([1.0, 1.0, dd]) @ U_.T
            self.local[a0:a1] = body
            self.mass[k], self.I[k], self.R[k] = mk.sum(), ev, com
            self.q[k] = matrix_to_quaternion(Rk)
        self.mol = np.asarray(system.mol)
        # momenta of the rigid part of the atom velocities (rigid.py:235-265)
        vel = np.asarray(vel, float)
        x = self.positions()
        self.P = np.zeros((M, 3))
        np.add.at(self.P, self.mol, m[:, None] * vel)
        Ls = np.zeros((M, 3))
        np.add.at(Ls, self.mol, m[:, None] * np.cross(x - self.R[self.mol], vel))
        Lb = np.einsum("kji,kj->ki", rotation_matrix(self.q), Ls)  # space -> body: R^T L
        self.p = 2.0 * quat_mul(self.q, np.concatenate([np.zeros((M, 1)), Lb], 1))
        self.F, self.epot = force_fn(x)
        self.step_count = 0

    def positions(self):
        Rm = rotation_matrix(self.q)[self.mol]
        return self.R[self.mol] + np.einsum("nij,nj->ni", Rm, self.local)

    def _kick(self, h: float) -> None:
        """p += h F: centre force and quaternion force 2 q (x) (0, body torque)."""
        M = self.sys.nmol
        x = self.positions()
        fc = np.zeros((M, 3))
        np.add.at(fc, self.mol, self.F)
        tau = np.zeros((M, 3))
        np.add.at(tau, self.mol, np.cross(x - self.R[self.mol], self.F))
        tb = np.einsum("kji,kj->ki", rotation_matrix(self.q), tau)
        self.P = self.P + h * fc
        self.p = self.p + h * 2.0 * quat_mul(self.q, np.concatenate([np.zeros((M, 1)), tb], 1))

    def _rotate(self, k: int, h: float) -> None:
        Pq = perm(k, self.q)
        zeta = h * np.sum(self.p * Pq, 1) / (4.0 * self.I[:, k - 1])
        c, s = np.cos(zeta)[:, None], np.sin(zeta)[:, None]
        Pp = perm(k, self.p)
        self.q = c * self.q + s * Pq
        self.p = c * self.p + s * Pp

    def free_rotor(self, h: float) -> None:
        self._rotate(3, 0.5 * h)
        self._rotate(2, 0.5 * h)
        self._rotate(1, h)
        self._rotate(2, 0.5 * h)
        self._rotate(3, 0.5 * h)

    def step(self, dt: float) -> None:
        self._kick(0.5 * dt)
        self.R = self.R + dt * self.P / self.mass[:, None]
        self.free_rotor(dt)
        self.F, self.epot = self.force_fn(self.positions())
        self._kick(0.5 * dt)
        self.step_count += 1

    def kinetic(self) -> float:
        """Translational P^2 / 2M plus rotational sum_k L_k^2 / 2 I_k, L_k = (P_k q) . p / 2."""
        L = np.stack([0.5 * np.sum(perm(k, self.q) * self.p, 1) for k in (1, 2, 3)], 1)
        return float(0.5 * np.sum(self.P**2 / self.mass[:, None]) + 0.5 * np.sum(L**2 / self.I))

    def temperature(self, nve: bool = True) -> float:
        """2 K / (dof kB), dof = 6 M - 3 in NVE (integrate.py:383)."""
        dof = 6 * self.sys.nmol - (3 if nve else 0)
        return 2.0 * self.kinetic() / (dof * KB)
