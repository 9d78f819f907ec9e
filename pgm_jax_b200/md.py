"""Rigid-molecule MD on the GPU with the pGM force field: the driver of the benchmarks.

The role of the reference's rigid-body engine (pgm_jax/md/simulation.py:55 Simulation with
md/integrate.py:743-761 _step and md/thermostats.py:195-240 Langevin): one step is
B A O A (forces) B on rigid bodies (B A (forces) B in NVE), run by the engine's kernels
(csrc/pgm_md.cu), with the force call in between.  A step is captured once into a CUDA graph (the CG loop as a device-side while
node) and replayed, so a step never returns to the host.

Units: nm, ps, amu, kJ/mol, K.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .forcefield import PGMForceField

KB = 0.0083144626181532  # kJ/mol/K (pgm_jax/units.py:16)


def _quat_from_matrix(R: np.ndarray) -> np.ndarray:
    """Unit quaternion (w, x, y, z), w >= 0, of a proper rotation matrix (Shepperd's method)."""
    t = np.trace(R)
    if t > 0:
        s = np.sqrt(t + 1.0) * 2
        q = [0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s]
    elif R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]:
        s = np.sqrt(1.0 + R[0, 0] - R[1, 1] - R[2, 2]) * 2
        q = [(R[2, 1] - R[1, 2]) / s, 0.25 * s, (R[0, 1] + R[1, 0]) / s, (R[0, 2] + R[2, 0]) / s]
    elif R[1, 1] > R[2, 2]:
        s = np.sqrt(1.0 + R[1, 1] - R[0, 0] - R[2, 2]) * 2
        q = [(R[0, 2] - R[2, 0]) / s, (R[0, 1] + R[1, 0]) / s, 0.25 * s, (R[1, 2] + R[2, 1]) / s]
    else:
        s = np.sqrt(1.0 + R[2, 2] - R[0, 0] - R[1, 1]) * 2
        q = [(R[1, 0] - R[0, 1]) / s, (R[0, 2] + R[2, 0]) / s, (R[1, 2] + R[2, 1]) / s, 0.25 * s]
    q = np.asarray(q)
    return q / np.linalg.norm(q) * (1.0 if q[0] >= 0 else -1.0)


def rigid_bodies(system, pos: np.ndarray, H: np.ndarray):
    """Centres of mass, quaternions, principal-frame coordinates and principal moments of every molecule.

    As pgm_jax/md/rigid.py:126-205: molecules are made whole (every atom at the minimum image of the
    first); the instances of one Molecule object share the principal frame of the first instance
    (moments ascending, a proper frame), and every instance's orientation is the Kabsch fit of that
    template to it.  Returns (com (M, 3), quat (M, 4), body (N, 3), inertia (M, 3)).
    """
    pos = np.asarray(pos, float)
    H = np.asarray(H, float)
    Hinv = np.linalg.inv(H)
    M = system.nmol
    com = np.zeros((M, 3))
    quat = np.zeros((M, 4))
    body = np.zeros((system.n, 3))
    inertia = np.zeros((M, 3))
    templates = {}
    for m in range(M):
        a0, a1 = system.mol_start[m], system.mol_start[m + 1]
        d = pos[a0:a1] - pos[a0]
        for _ in range(2):  # a second pass catches what a skewed box leaves after one rounding
            d = d - np.round(d @ Hinv) @ H
        x = pos[a0] + d
        w = system.masses[a0:a1]
        c = (w[:, None] * x).sum(0) / w.sum()
        y = x - c
        key = id(system.molecules[m])
        if key not in templates:
            Itens = np.sum(w[:, None, None] * ((y * y).sum(1)[:, None, None] * np.eye(3) - y[:, :, None] * y[:, None, :]), 0)
            ev, V = np.linalg.eigh(Itens)
            if np.linalg.det(V) < 0:
                V[:, 0] = -V[:, 0]
            templates[key] = (y @ V, ev)
        b, ev = templates[key]
        U, _, Vt = np.linalg.svd(b.T @ y)  # Kabsch: y ~ b @ R.T
        dd = np.sign(np.linalg.det(Vt.T @ U.T))
        R = Vt.T @ np.diag([1.0, 1.0, dd]) @ U.T
        com[m] = c
        quat[m] = _quat_from_matrix(R)
        body[a0:a1] = b
        inertia[m] = ev
    return com, quat, body, inertia


def rigid_momenta(system, pos: np.ndarray, com: np.ndarray, quat: np.ndarray, vel: np.ndarray):
    """Linear momenta P (M, 3) and body-frame angular momenta L (M, 3) of the rigid part of atom
    velocities (rigid.py:235-265): P_k = sum m v, L_k = R_k^T sum m (r - X_k) x v, r the atoms of
    the bodies."""
    m = np.asarray(system.masses, float)
    mol = np.asarray(system.mol)
    P = np.zeros((system.nmol, 3))
    np.add.at(P, mol, m[:, None] * vel)
    L = np.zeros((system.nmol, 3))
    np.add.at(L, mol, m[:, None] * np.cross(pos - com[mol], vel))
    w, x, y, z = quat.T
    Rm = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)
    return P, np.einsum("kji,kj->ki", Rm, L)


def _rot(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


class RigidMD:
    """Langevin (gamma > 0) or NVE rigid-body MD of a PGMForceField's systems on the GPU.

        md = RigidMD(ff, pos, H, temperature=298.0, dt_fs=1.0, gamma_ps=2.0, seed=1)
        md.run(100)                      # steps (graph replays)
        md.temperature(), md.energy()

    Momenta are drawn at `temperature` (seeded, no net momentum), or, with `velocities` (N, 3)
    [nm/ps], taken from the rigid part of those atom velocities.  NVE (gamma_ps = 0) is the
    reference's velocity Verlet: kick, one drift of dt, forces, kick.
    """

    def __init__(self, ff: PGMForceField, pos, H, temperature=298.0, dt_fs: float = 1.0, gamma_ps: float = 0.0,
                 seed: int = 1, velocity_seed: int | None = None, velocities=None) -> None:
        self.ff = ff
        self.dev = ff.device
        self.dt = dt_fs * 1e-3
        self.gamma = float(gamma_ps)
        self.seed = int(seed)
        self.step_count = 0
        systems = ff.systems
        H = np.asarray(H, float)
        boxes = H if H.ndim == 3 else np.stack([H] * ff.nsys)
        temps = np.broadcast_to(np.asarray(temperature, float), (ff.nsys,)).copy()
        pos = np.asarray(pos, float)
        coms, quats, bodies, inertias, msys, mstart, masses = [], [], [], [], [], [0], []
        for k, sy in enumerate(systems):
            sl = slice(int(ff.offsets[k]), int(ff.offsets[k + 1]))
            c, q, b, I = rigid_bodies(sy, pos[sl], boxes[k])
            coms.append(c); quats.append(q); bodies.append(b); inertias.append(I)
            msys.append(np.full(sy.nmol, k, np.int32))
            mstart.extend((np.asarray(sy.mol_start[1:]) + ff.offsets[k]).tolist())
            masses.append(sy.masses)
        com = np.concatenate(coms); quat = np.concatenate(quats); body = np.concatenate(bodies)
        inertia = np.concatenate(inertias); msys = np.concatenate(msys); masses = np.concatenate(masses)
        mstart = np.asarray(mstart, np.int32)
        self.nmol = len(com)
        self.temps = temps
        self.kT = torch.tensor(KB * temps, dtype=torch.float64, device=self.dev)
        # Maxwell momenta at each system's temperature
        rng = np.random.default_rng(seed if velocity_seed is None else velocity_seed)
        mt = np.add.reduceat(masses, mstart[:-1])
        kTm = KB * temps[msys]
        P = rng.normal(size=(self.nmol, 3)) * np.sqrt(mt * kTm)[:, None]
        L = rng.normal(size=(self.nmol, 3)) * np.sqrt(inertia * kTm[:, None])
        for k in range(ff.nsys):  # no net momentum per system
            sel = msys == k
            P[sel] -= P[sel].mean(0)
        if velocities is not None:  # the rigid part of given atom velocities [nm/ps] (Simulation(velocities=...))
            vel = np.asarray(velocities, float).reshape(ff.n, 3)
            for k, sy in enumerate(systems):
                sl = slice(int(ff.offsets[k]), int(ff.offsets[k + 1]))
                sel = msys == k
                R = np.stack([np.asarray(_rot(q)) for q in quat[sel]])
                bpos = com[sel][sy.mol] + np.einsum("nij,nj->ni", R[sy.mol], body[sl])
                P[sel], L[sel] = rigid_momenta(sy, bpos, com[sel], quat[sel], vel[sl])
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=self.dev)  # noqa: E731
        self.com, self.quat, self.mom, self.angmom = t(com), t(quat), t(P), t(L)
        self.box = t(boxes)
        self.pos = t(pos)
        self.ind = ff.init_induction()
        self.forces = torch.zeros((ff.n, 3), dtype=torch.float64, device=self.dev)
        lib = _lib.load()
        self._lib = lib
        self.stream = torch.cuda.Stream(self.dev)  # a non-default stream: steps are captured into graphs
        self._keep = [np.ascontiguousarray(a) for a in (mstart, msys, masses, body, inertia)]
        h = C.c_void_p()
        _lib.check(lib.pgm_rigid_create(self.nmol, *[C.c_void_p(a.ctypes.data) for a in self._keep], ff.device.index or 0,
                                        C.byref(h)))
        self._h = h
        self._graph = None
        self.result = None
        self._first_forces()

    def _stream(self):
        return C.c_void_p(self.stream.cuda_stream)

    def _first_forces(self) -> None:
        # positions from the rigid bodies, then forces (the reference's integrator init)
        with torch.cuda.stream(self.stream):
            _lib.check(self._lib.pgm_rigid_begin_step(self._h, self._stream(), 0.0, 0.0, None, 0, None, _p(self.com),
                                                      _p(self.quat), _p(self.mom), _p(self.angmom), _p(self.pos), _p(self.box)))
            self.result = self.ff.compute_into(self.pos, self.box, self.ind, self.forces)
        self.stream.synchronize()

    def _step_enqueue(self) -> None:
        st = self._stream()
        lib = self._lib
        with torch.cuda.stream(self.stream):
            _lib.check(lib.pgm_rigid_begin_step(self._h, st, self.dt, self.gamma, _p(self.kT), self.seed, _p(self.forces),
                                                _p(self.com), _p(self.quat), _p(self.mom), _p(self.angmom), _p(self.pos),
                                                _p(self.box)))
            self.result = self.ff.compute_into(self.pos, self.box, self.ind, self.forces)
            _lib.check(lib.pgm_rigid_end_step(self._h, st, self.dt, _p(self.forces), _p(self.quat), _p(self.mom),
                                              _p(self.angmom)))

    def step(self) -> None:
        """One MD step, launched directly (the CG loop driven from the host)."""
        self._step_enqueue()
        self.step_count += 1

    def capture(self) -> None:
        """Capture one step into a CUDA graph (CG loop as a device-side while node); a graph captured
        before is released."""
        self.stream.synchronize()
        if self._graph is not None:
            _lib.check(self._lib.pgm_graph_destroy(self._graph))
            self._graph = None
        st = self._stream()
        _lib.check(self._lib.pgm_graph_begin(st))
        ex = C.c_void_p()
        try:
            self._step_enqueue()
        except Exception:
            self._lib.pgm_graph_end(st, C.byref(ex))  # close the capture; the error is the one raised
            if ex.value:
                self._lib.pgm_graph_destroy(ex)
            raise
        _lib.check(self._lib.pgm_graph_end(st, C.byref(ex)))
        self._graph = ex
        self.launches_per_iteration = int(self._lib.pgm_launches_per_iteration(self.ff._h))
        self.unrolled_iterations = int(self._lib.pgm_unrolled_iterations(self.ff._h))
        # launches of a replay: these + max(unrolled, CG iterations) x launches_per_iteration
        self.launches_outside_loop = (self.ff.last_launch_count() + 2
                                      - (1 + self.unrolled_iterations) * self.launches_per_iteration)

    def run(self, n: int) -> None:
        """n steps: graph replays when captured, else direct launches."""
        for _ in range(n):
            if self._graph is not None:
                _lib.check(self._lib.pgm_graph_launch(self._graph, self._stream()))
            else:
                self._step_enqueue()
            self.step_count += 1

    def set_temperatures(self, temps) -> None:
        """Thermostat temperature of every system [K] (written in place: captured steps see it)."""
        temps = np.broadcast_to(np.asarray(temps, float), (self.ff.nsys,)).copy()
        self.temps = temps
        with torch.cuda.stream(self.stream):
            self.kT.copy_(torch.tensor(KB * temps, dtype=torch.float64), non_blocking=False)

    def scale_momenta(self, factors) -> None:
        """Linear and angular momenta of every system's molecules times its factor (on the MD stream)."""
        f = torch.tensor(np.broadcast_to(np.asarray(factors, float), (self.ff.nsys,)).copy(), dtype=torch.float64,
                         device=self.dev)
        with torch.cuda.stream(self.stream):
            _lib.check(self._lib.pgm_rigid_scale_momenta(self._h, self._stream(), _p(f), _p(self.mom), _p(self.angmom)))
        self.stream.synchronize()

    def kinetic(self) -> np.ndarray:
        ke = torch.zeros(self.ff.nsys, dtype=torch.float64, device=self.dev)
        self.stream.wait_stream(torch.cuda.current_stream(self.dev))
        _lib.check(self._lib.pgm_rigid_kinetic(self._h, self._stream(), _p(self.mom), _p(self.angmom), _p(ke)))
        self.stream.synchronize()
        return ke.cpu().numpy()

    def energy(self) -> dict:
        """Energies of the last force call (elec, vdw, total per system) and the kinetic energy."""
        self.stream.synchronize()
        r = self.result
        return {"elec": r.energy["elec"].cpu().numpy(), "vdw": r.energy["vdw"].cpu().numpy(),
                "total": r.energy["total"].cpu().numpy(), "kinetic": self.kinetic()}

    def temperature(self) -> np.ndarray:
        """Instantaneous temperature per system (6 degrees of freedom per rigid molecule minus 3)."""
        nm = np.array([sy.nmol for sy in self.ff.systems])
        return 2.0 * self.kinetic() / ((6 * nm - 3) * KB)

    def __del__(self) -> None:
        try:
            if getattr(self, "_graph", None) is not None:
                self._lib.pgm_graph_destroy(self._graph)
            if getattr(self, "_h", None) is not None and self._h.value:
                self._lib.pgm_rigid_destroy(self._h)
        except Exception:
            pass


def _p(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())
