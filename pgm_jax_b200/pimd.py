"""Path-integral MD (PIMD with the PILE-L thermostat, thermostatted RPMD, RPMD) of flexible pGM
water on the GPU.

The reference's PIMDIntegrator / RingPolymer / PILEStep / PGMBeads (pgm_jax/md/pimd.py:135-1159):
P beads per atom sampled classically at P T with springs m omega_P^2 |q^k - q^(k+1)|^2 / 2,
omega_P = P kB T / hbar; BAOAB with the free ring polymer in normal modes (Cayley steps) and
Langevin on every mode (internal modes gamma_l = 2 lam omega_l, the centroid 1 / tau_centroid).
Here the P beads are the P systems of one batched force field (csrc/pgm_api.cu), so every bead's
rows, PME and induced-dipole solve (each bead with its own induction history) run in the same
kernel launches, and the integrator is csrc/pgm_pimd.cu (one warp per atom component, beads in
lanes).  The intramolecular surface is q-TIP4P/F (the reference's flexible water,
pgm_jax/models/water.py:33-69); the intramolecular pGM terms (Gaussian monopoles and covalent
dipoles of the molecule) come from the force field for any geometry.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from .forcefield import MDSettings, PGMForceField

KB = 0.0083144626181532  # kJ/mol/K (pgm_jax/units.py:16)
HBAR = 0.0635077993  # kJ/mol ps (pgm_jax/units.py:20)
KCAL = 4.184
# q-TIP4P/F (Habershon, Markland and Manolopoulos, J. Chem. Phys. 131, 024501 (2009)), as
# pgm_jax/models/water.py:33: D [kJ/mol], alpha [1/nm], r_eq [nm], k_theta [kJ/mol/rad^2], theta_eq [deg]
QTIP4PF = {"D": 116.09 * KCAL, "alpha": 22.87, "r_eq": 0.09419, "k_theta": 87.85 * KCAL, "theta_eq": 107.4}


def normal_modes(P: int) -> tuple[np.ndarray, np.ndarray]:
    """(C (P, P), idx (P,)): C[j, l] of bead j and mode l, real orthonormal, ordered by frequency --
    the centroid 1/sqrt(P), then sqrt(2/P) cos and sin (2 pi j l / P) pairs, then (-1)^j / sqrt(P)
    for even P -- and the frequency index of every mode (pimd.py:135-162)."""
    P = int(P)
    j = np.arange(P, dtype=float)
    cols, idx = [np.full(P, 1.0 / math.sqrt(P))], [0]
    for l in range(1, (P - 1) // 2 + 1):
        ang = 2.0 * math.pi * j * l / P
        cols += [math.sqrt(2.0 / P) * np.cos(ang), math.sqrt(2.0 / P) * np.sin(ang)]
        idx += [l, l]
    if P % 2 == 0 and P > 1:
        cols.append(np.where(np.arange(P) % 2 == 0, 1.0, -1.0) / math.sqrt(P))
        idx.append(P // 2)
    return np.stack(cols, 1), np.asarray(idx, int)


class RingPolymer:
    """Normal modes and mode frequencies of P beads at T (pimd.py:183-236)."""

    def __init__(self, beads: int, temperature: float) -> None:
        self.P = int(beads)
        if self.P < 1:
            raise ValueError("at least one bead")
        self.T = float(temperature)
        self.kT = KB * self.T
        self.kT_P = self.P * self.kT
        self.omega_P = self.kT_P / HBAR
        self.C, idx = normal_modes(self.P)
        self.omega = 2.0 * self.omega_P * np.sin(np.pi * idx / self.P)
        self.omega[0] = 0.0

    def spring(self, q: np.ndarray, mass: np.ndarray) -> np.ndarray:
        """sum_k m omega_P^2 |q^k - q^(k+1)|^2 / 2 per atom; q (P, N, 3), mass (N,)."""
        d = q - np.roll(q, -1, axis=0)
        return 0.5 * self.omega_P**2 * mass * np.sum(d * d, axis=(0, 2))


def frictions(ring: RingPolymer, mode: str = "pimd", tau_centroid: float = 0.2, lam: float | None = None,
              centroid: str = "l") -> np.ndarray:
    """Friction of every mode [1/ps] (PILEStep, pimd.py:375-397): 2 lam omega_l on the internal
    modes (lam 1 for "pimd", 1/2 for "trpmd"), 1/tau_centroid on the centroid for "pimd" with the
    Langevin centroid (PILE-L, centroid "l"), 0 with Bussi's (PILE-G, centroid "g"), none for
    "rpmd"."""
    mode = mode.lower()
    if mode not in ("pimd", "trpmd", "rpmd"):
        raise ValueError(f"mode: 'pimd' | 'trpmd' | 'rpmd', not {mode!r}")
    if centroid not in ("l", "g"):
        raise ValueError(f"centroid thermostat must be 'l' (Langevin) or 'g' (Bussi), not {centroid!r}")
    if tau_centroid <= 0:
        raise ValueError("tau_centroid must be > 0")
    lam = (0.5 if mode == "trpmd" else 1.0) if lam is None else float(lam)
    g = 2.0 * lam * ring.omega
    g[0] = 1.0 / tau_centroid if (mode == "pimd" and centroid == "l") else 0.0
    if mode == "rpmd":
        g[:] = 0.0
    return g


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


class PIMD:
    """Ring-polymer MD of one flexible system: P beads as a batch of the force field.

    system, pos (N, 3) [nm], H (3, 3) [nm]; settings an MDSettings (pme_grid etc.); beads P <= 32.
    The beads start on the free ring polymer around `pos` (seeded) with momenta at P kB T.
    mode "pimd" (PILE-L, or PILE-G with centroid="g": Bussi's rescaling of the centroid with time
    constant tau_centroid), "trpmd" or "rpmd" (no thermostat).  Water molecules (3 atoms: O, H, H)
    get the q-TIP4P/F intramolecular term.
    """

    def __init__(self, system, pos, H, settings: MDSettings, beads: int = 32, temperature: float = 300.0, dt_fs: float = 0.5,
                 mode: str = "pimd", tau_centroid: float = 0.2, lam: float | None = None, seed: int = 1, device: int = 0,
                 pme_grid=None, bonded: dict | None = QTIP4PF, centroid: str = "l") -> None:
        if not 1 <= int(beads) <= 32:
            raise ValueError("1 <= beads <= 32")
        self.P = int(beads)
        self.ring = RingPolymer(self.P, temperature)
        self.mode = mode
        self.dt = dt_fs * 1e-3
        self.seed = int(seed)
        H = np.asarray(H, float)
        grids = None if pme_grid is None else [tuple(pme_grid)] * self.P
        self.ff = PGMForceField([system] * self.P, [H] * self.P, settings, pme_grids=grids, device=device)
        self.dev = self.ff.device
        self.n = system.n
        self.mass_np = np.asarray(system.masses, float)
        t = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device=self.dev)  # noqa: E731
        rng = np.random.default_rng(seed)
        # beads on the free ring polymer around pos: internal mode l ~ N(0, kT_P / (m omega_l^2))
        y = np.zeros((self.P, self.n, 3))
        y[0] = math.sqrt(self.P) * np.asarray(pos, float)
        for l in range(1, self.P):
            y[l] = rng.normal(size=(self.n, 3)) * np.sqrt(self.ring.kT_P / self.mass_np)[:, None] / self.ring.omega[l]
        q = np.einsum("jl,lnc->jnc", self.ring.C, y)
        p = rng.normal(size=(self.P, self.n, 3)) * np.sqrt(self.mass_np * self.ring.kT_P)[None, :, None]
        self.q = t(q.reshape(-1, 3))
        self.p = t(p.reshape(-1, 3))
        self.box = t(np.stack([H] * self.P))
        self.forces = torch.zeros_like(self.q)
        self.C = t(self.ring.C)
        self.omega = t(self.ring.omega)
        self.gamma = t(frictions(self.ring, mode, tau_centroid, lam, centroid))
        self.tau0 = float(tau_centroid)
        self.centroid_bussi = mode == "pimd" and centroid == "g"
        self.bussi_work = torch.zeros(4, dtype=torch.float64, device=self.dev)  # K, alpha, R1, S of the last step
        self.mass = t(self.mass_np)
        self.counter = torch.zeros(1, dtype=torch.int64, device=self.dev)
        self.ind = self.ff.init_induction()
        waters = [m for m in range(system.nmol) if system.mol_start[m + 1] - system.mol_start[m] == 3]
        self.bonded = None
        if bonded and waters:
            first = np.concatenate([np.asarray(system.mol_start)[waters] + k * self.n for k in range(self.P)]).astype(np.int32)
            msys = np.repeat(np.arange(self.P, dtype=np.int32), len(waters))
            self.bonded = (t(first, torch.int32), t(msys, torch.int32),
                           np.array([bonded["D"], bonded["alpha"], bonded["r_eq"], bonded["k_theta"],
                                     math.radians(bonded["theta_eq"])], float))
        self.e_bond = torch.zeros(self.P, dtype=torch.float64, device=self.dev)
        self._lib = _lib.load()
        self.stream = torch.cuda.Stream(self.dev)
        self._graph = None
        self.result = None
        with torch.cuda.stream(self.stream):
            self._forces()
        self.stream.synchronize()

    def _st(self):
        return C.c_void_p(self.stream.cuda_stream)

    def _forces(self) -> None:
        self.result = self.ff.compute_into(self.q, self.box, self.ind, self.forces)
        if self.bonded is not None:
            first, msys, prm = self.bonded
            self.e_bond.zero_()
            _lib.check(self._lib.pgm_water_bonded(self._st(), int(first.numel()), _p(first), _p(msys), _p(self.q),
                                                  C.c_void_p(prm.ctypes.data), _p(self.forces), _p(self.e_bond)))

    def _step_enqueue(self) -> None:
        lib, st, h = self._lib, self._st(), 0.5 * self.dt
        n3 = 3 * self.P * self.n
        with torch.cuda.stream(self.stream):
            _lib.check(lib.pgm_pimd_kick(st, n3, h, _p(self.forces), _p(self.p)))
            scale = None
            if self.centroid_bussi:  # PILE-G: the centroid's Bussi factor from the momenta before the O step
                _lib.check(lib.pgm_pimd_centroid_bussi(st, self.P, self.n, _p(self.C), _p(self.mass), self.dt, self.ring.kT_P,
                                                       self.tau0, self.seed, _p(self.counter), _p(self.p), _p(self.bussi_work)))
                scale = C.c_void_p(self.bussi_work.data_ptr() + 8)
            _lib.check(lib.pgm_pimd_free_thermostat_scaled(st, self.P, self.n, _p(self.C), _p(self.omega), _p(self.gamma),
                                                           _p(self.mass), self.dt, self.ring.kT_P, self.seed, _p(self.counter),
                                                           _p(self.q), _p(self.p), scale))
            self._forces()
            _lib.check(lib.pgm_pimd_kick(st, n3, h, _p(self.forces), _p(self.p)))

    def step(self) -> None:
        """One step, launched directly."""
        self._step_enqueue()

    def capture(self) -> None:
        """Capture one step into a CUDA graph (the solver's loop as a device-side while node)."""
        self.stream.synchronize()
        st = self._st()
        _lib.check(self._lib.pgm_graph_begin(st))
        ex = C.c_void_p()
        try:
            self._step_enqueue()
        except Exception:
            self._lib.pgm_graph_end(st, C.byref(ex))
            if ex.value:
                self._lib.pgm_graph_destroy(ex)
            raise
        _lib.check(self._lib.pgm_graph_end(st, C.byref(ex)))
        self._graph = ex

    def run(self, n: int) -> None:
        for _ in range(n):
            if self._graph is not None:
                _lib.check(self._lib.pgm_graph_launch(self._graph, self._st()))
            else:
                self._step_enqueue()

    def estimators(self) -> dict:
        """Estimators of the current state (pimd.py:704-736): per-atom primitive ("prim") and
        centroid-virial ("cv") kinetic energies summed over atoms [kJ/mol], the bead kinetic
        energy, spring energy, potential U (all beads: force field + bonded), the ring-polymer
        Hamiltonian H_P, the normal-mode temperatures [K] and the centroid's."""
        self.stream.synchronize()
        P, n, ring = self.P, self.n, self.ring
        q = self.q.cpu().numpy().reshape(P, n, 3)
        p = self.p.cpu().numpy().reshape(P, n, 3)
        f = self.forces.cpu().numpy().reshape(P, n, 3)
        m = self.mass_np
        U = float(self.result.energy["total"].sum()) + float(self.e_bond.sum())
        spring = ring.spring(q, m)
        qc = q.mean(0)
        prim = 1.5 * P * ring.kT - spring / P
        cv = 1.5 * ring.kT - 0.5 / P * np.sum((q - qc[None]) * f, axis=(0, 2))
        ke = 0.5 * np.sum(p * p / m[None, :, None])
        pn = np.einsum("jl,jnc->lnc", ring.C, p)
        t_modes = np.sum(pn * pn / m[None, :, None], axis=(1, 2)) / (3.0 * n * KB * P)
        return {"prim": float(prim.sum()), "cv": float(cv.sum()), "ke_beads": ke, "spring": float(spring.sum()), "upot": U,
                "hamiltonian": ke + float(spring.sum()) + U, "t_modes": t_modes, "t_centroid": float(t_modes[0]),
                "epot": U / P}

    def __del__(self) -> None:
        try:
            if getattr(self, "_graph", None) is not None:
                self._lib.pgm_graph_destroy(self._graph)
        except Exception:
            pass
