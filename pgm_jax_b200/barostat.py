"""Isotropic Monte Carlo barostat for the rigid-molecule MD driver (NPT).

The reference's barostat (`pgm_jax/md/barostats.py:26-60` settings, the move in
`Integrator._barostat`, `pgm_jax/md/integrate.py:763-817`): every `every` steps one volume move,
dV uniform in [-dv, dv]; molecular centres and box scaled by s = (V'/V)^(1/3), orientations and
momenta kept; the trial energy (dipoles re-solved from the current ones, no history push) is
accepted with probability min(1, exp(-w / kT)),

    w = (E' - E) + P dV - M kT ln(V'/V)        (M molecules of the system);

accepted moves take the trial box, centres and dipoles and recompute the forces.  After every 10
tries the step size dv is divided by 1.1 below 25 % acceptance and multiplied by 1.1 above 75 %
(at most 0.3 V); it starts at 0.01 V.

Here every system of a batch (replicas, uneven boxes) makes its own move, and one trial-energy
evaluation (`PGMForceField.energy`, one launch per kernel for the batch) serves them all.  The
decision and the step-size rule are plain functions of host arrays (`mc_accept`, `mc_adapt`).
"""

from __future__ import annotations

import numpy as np
import torch

KJMOL_NM3_PER_BAR = 1.0 / 16.605390671738466  # 1 bar in kJ/mol/nm^3 (pgm_jax/units.py:18)


def mc_accept(e_new, e_old, dV, V, nmol, kT, pressure, log_u) -> np.ndarray:
    """Metropolis test of volume moves (integrate.py:799-800); all arguments per system, pressure
    in kJ/mol/nm^3, log_u the log of a uniform number.  A move to V' <= 0 is rejected."""
    e_new, e_old, dV, V = (np.asarray(a, float) for a in (e_new, e_old, dV, V))
    Vn = V + dV
    w = (e_new - e_old) + pressure * dV - np.asarray(nmol, float) * np.asarray(kT, float) * np.log(np.maximum(Vn, 1e-12) / V)
    with np.errstate(invalid="ignore"):
        return (Vn > 0) & np.isfinite(e_new) & (np.asarray(log_u, float) < -w / np.asarray(kT, float))


def mc_adapt(dv, tries, accepted, V):
    """The step-size rule after a move (integrate.py:809-817): returns (dv, tries, accepted) with
    the window counters reset once 10 tries have been made."""
    dv, tries, accepted, V = (np.asarray(a, float).copy() for a in (dv, tries, accepted, V))
    window = tries >= 10
    rate = accepted / np.maximum(tries, 1)
    dv = np.where(window & (rate < 0.25), dv / 1.1, np.where(window & (rate > 0.75), dv * 1.1, dv))
    dv = np.minimum(dv, 0.3 * V)
    tries = np.where(window, 0, tries)
    accepted = np.where(window, 0, accepted)
    return dv, tries.astype(int), accepted.astype(int)


class MonteCarloBarostat:
    """NPT for a `RigidMD`: `run(n)` advances n steps with a volume move every `every` steps.

    pressure in bar (one value or one per system); seed of the move's uniform numbers.
    """

    def __init__(self, md, pressure: float = 1.0, every: int = 100, seed: int = 0) -> None:
        if int(every) < 1:
            raise ValueError("every must be >= 1")
        p = np.broadcast_to(np.asarray(pressure, float), (md.ff.nsys,)).copy()
        if not np.all(np.isfinite(p)):
            raise ValueError("pressure must be finite")
        self.md = md
        self.every = int(every)
        self.pressure = p * KJMOL_NM3_PER_BAR
        self.rng = np.random.default_rng(seed)
        ff = md.ff
        mstart, msys = md._keep[0], md._keep[1]
        self.nmol = np.bincount(msys, minlength=ff.nsys)
        # atom -> molecule and atom -> system maps on the device (molecular scaling of positions)
        atom_mol = np.repeat(np.arange(len(mstart) - 1), np.diff(mstart))
        self._atom_mol = torch.tensor(atom_mol, dtype=torch.int64, device=md.dev)
        self._atom_sys = torch.tensor(msys[atom_mol], dtype=torch.int64, device=md.dev)
        self._mol_sys = torch.tensor(msys, dtype=torch.int64, device=md.dev)
        self.dv = 0.01 * self.volumes()
        self.tries = np.zeros(ff.nsys, int)
        self.accepted = np.zeros(ff.nsys, int)
        self.total_tries = np.zeros(ff.nsys, int)
        self.total_accepted = np.zeros(ff.nsys, int)

    def volumes(self) -> np.ndarray:
        return np.abs(np.linalg.det(self.md.box.cpu().numpy()))

    def attempt(self, dV=None, log_u=None) -> np.ndarray:
        """One volume move for every system (dV and log_u drawn when not given); returns the
        per-system acceptance."""
        md, ff = self.md, self.md.ff
        md.stream.synchronize()
        H = md.box.cpu().numpy()
        V = np.abs(np.linalg.det(H))
        S = ff.nsys
        if dV is None:
            dV = (2.0 * self.rng.uniform(size=S) - 1.0) * self.dv
        if log_u is None:
            log_u = np.log(self.rng.uniform(size=S))
        dV = np.broadcast_to(np.asarray(dV, float), (S,))
        log_u = np.broadcast_to(np.asarray(log_u, float), (S,))
        s = np.cbrt(np.maximum(V + dV, 1e-12) / V)
        st = torch.tensor(s, dtype=torch.float64, device=md.dev)
        with torch.cuda.stream(md.stream):
            e_old = md.result.energy["total"].clone()
            # centres scaled, orientations kept: every atom moves by (s - 1) times its molecule's centre
            shift = (st[self._atom_sys] - 1.0)[:, None] * md.com[self._atom_mol]
            pos_n = md.pos + shift
            box_n = md.box * st[:, None, None]
            e_new, ind_n, _, ovf = ff.energy(pos_n, box_n, None, md.ind)
            md.stream.synchronize()
        e_new_h = e_new.cpu().numpy().copy()
        e_new_h[ovf.cpu().numpy()] = np.nan  # a trial that overflowed its rows is rejected
        kT = md.kT.cpu().numpy()
        acc = mc_accept(e_new_h, e_old.cpu().numpy(), dV, V, self.nmol, kT, self.pressure, log_u)
        if acc.any():
            a = torch.tensor(acc, device=md.dev)
            with torch.cuda.stream(md.stream):
                atoms = a[self._atom_sys]
                md.pos.copy_(torch.where(atoms[:, None], pos_n, md.pos))
                md.com.copy_(torch.where(a[self._mol_sys][:, None], md.com * st[self._mol_sys][:, None], md.com))
                md.box.copy_(torch.where(a[:, None, None], box_n, md.box))
                md.ind.mu.copy_(torch.where(atoms[:, None], ind_n.mu, md.ind.mu))
                # forces of the new state (the whole batch: a system that kept its state is
                # evaluated again at the same positions)
                md.result = ff.compute_into(md.pos, md.box, md.ind, md.forces)
            md.stream.synchronize()
        self.tries += 1
        self.accepted += acc.astype(int)
        self.total_tries += 1
        self.total_accepted += acc.astype(int)
        self.dv, self.tries, self.accepted = mc_adapt(self.dv, self.tries, self.accepted, self.volumes())
        return acc

    def run(self, n: int) -> None:
        """n MD steps (graph replays when the MD is captured) with a move after every `every`."""
        done = 0
        while done < n:
            k = min(self.every - md_phase(self.md.step_count, self.every), n - done)
            self.md.run(k)
            done += k
            if self.md.step_count % self.every == 0:
                self.attempt()


def md_phase(step_count: int, every: int) -> int:
    """Steps since the last move boundary."""
    return step_count % every
