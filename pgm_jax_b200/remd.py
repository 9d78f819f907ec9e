"""Temperature replica exchange (parallel tempering) over the systems of one batched engine.

The reference (pgm_jax/md/remd.py) runs R copies of a system at the temperatures of a ladder and,
every `exchange_every` steps, tries to swap the configurations of neighbouring temperatures,
alternately the even pairs (0,1), (2,3), ... and the odd pairs (1,2), ... (remd.py:161-181), with
the Metropolis probability min(1, exp(-Delta)), Delta = u_i(x_j) + u_j(x_i) - u_i(x_i) - u_j(x_j)
and u_k(x) = U(x) / (kB T_k) (remd.py:184-256); the momenta of an exchanged configuration are
rescaled by sqrt(T_new / T_old).

Here all replicas are systems of one batch (one engine launch per kernel for all of them,
csrc/pgm_api.cu), and an accepted swap moves the two temperatures instead of the two
configurations: the thermostat temperature of each system is a device array read by the captured
step, the momenta are rescaled on the GPU (pgm_rigid_scale_momenta), and nothing else moves.  The
walkers (configurations) and their round trips are tracked exactly as in the reference.  Across
ranks (one process per GPU, each holding some of the replicas) the only exchange of data is an
all-gather of the potential energies per exchange; every rank draws the same uniforms and takes the
same decisions.
"""

from __future__ import annotations

from typing import Sequence

import numpy as np

KB = 0.0083144626181532  # kJ/mol/K (pgm_jax/units.py:16)


def geometric_ladder(t_min: float, t_max: float, n: int) -> np.ndarray:
    """n temperatures t_min (t_max / t_min)^(k / (n - 1)) [K] (remd.py:127-158); ValueError unless
    n >= 2 and 0 < t_min < t_max."""
    if int(n) < 2 or not (0.0 < t_min < t_max):
        raise ValueError(f"a temperature ladder takes at least 2 rungs and 0 < t_min < t_max (got n={n}, {t_min}, {t_max})")
    k = np.arange(int(n), dtype=float)
    return float(t_min) * np.exp(np.log(float(t_max) / float(t_min)) * k / (int(n) - 1))


def exchange_pairs(n: int, parity: int) -> list[tuple[int, int]]:
    """The disjoint neighbour pairs of an exchange round: (0,1), (2,3), ... when parity is even,
    (1,2), (3,4), ... when odd (remd.py:161-181)."""
    return [(i, i + 1) for i in range(int(parity) & 1, int(n) - 1, 2)]


def temperature_reduced_energies(temperatures, U, V=None, pressure: float | None = None) -> np.ndarray:
    """u[i, j] = (U_j + P V_j) / (kB T_i) (remd.py:231-256)."""
    beta = 1.0 / (KB * np.asarray(temperatures, float))
    H = np.asarray(U, float) if pressure is None else np.asarray(U, float) + float(pressure) * np.asarray(V, float)
    return np.outer(beta, H)


def metropolis(u, pairs: Sequence[tuple[int, int]], uniforms) -> tuple[np.ndarray, np.ndarray]:
    """Accept or reject the swaps of disjoint pairs (remd.py:184-228).

    u[i, j]: reduced energy in state i of the configuration now in state j.  Returns (accepted per
    pair, src) with state i holding afterwards the configuration previously in state src[i].
    ValueError for pairs that are not disjoint; FloatingPointError for a non-finite Delta."""
    u = np.asarray(u, float)
    src = np.arange(u.shape[0])
    accepted = np.zeros(len(pairs), bool)
    used: set[int] = set()
    for k, (i, j) in enumerate(pairs):
        if i == j or i in used or j in used:
            raise ValueError(f"replica {i} or {j} appears in two exchange pairs of one attempt")
        used.add(i)
        used.add(j)
        delta = (u[i, j] - u[i, i]) + (u[j, i] - u[j, j])
        if not np.isfinite(delta):
            raise FloatingPointError(f"exchange {i}-{j}: reduced energy difference {delta}")
        accepted[k] = bool(delta <= 0.0 or uniforms[k] < np.exp(-delta))
        if accepted[k]:
            src[i], src[j] = src[j], src[i]
    return accepted, src


class ExchangeStatistics:
    """Attempts and acceptances per pair of states, the walker (configuration) at each state, and
    each walker's one-way transits between the ends of the ladder and round trips (lowest ->
    highest -> lowest), as remd.py:259-358 counts them."""

    def __init__(self, n: int) -> None:
        self.n = int(n)
        self.attempts = np.zeros((self.n, self.n), int)
        self.accepts = np.zeros((self.n, self.n), int)
        self.replica = np.arange(self.n)
        self.last_end = np.full(self.n, -1)  # per walker: 0 lowest, 1 highest, -1 none yet
        self.phase = np.zeros(self.n, int)  # per walker: 1 after the lowest end, 2 after lowest then highest
        self.round_trips = np.zeros(self.n, int)
        self.transits = np.zeros(self.n, int)
        self.n_exchanges = 0
        self._visit_ends()

    def _visit_ends(self) -> None:
        lo, hi = int(self.replica[0]), int(self.replica[-1])
        if self.last_end[lo] == 1:
            self.transits[lo] += 1
        if self.phase[lo] == 2:
            self.round_trips[lo] += 1
        self.last_end[lo], self.phase[lo] = 0, 1
        if self.last_end[hi] == 0:
            self.transits[hi] += 1
        if self.phase[hi] == 1:
            self.phase[hi] = 2
        self.last_end[hi] = 1

    def record(self, pairs, accepted, src) -> None:
        for (i, j), a in zip(pairs, accepted):
            self.attempts[i, j] += 1
            self.attempts[j, i] += 1
            if a:
                self.accepts[i, j] += 1
                self.accepts[j, i] += 1
        self.replica = self.replica[np.asarray(src)]
        self.n_exchanges += 1
        self._visit_ends()

    def acceptance(self) -> np.ndarray:
        return self.accepts / np.maximum(self.attempts, 1)

    def neighbour_acceptance(self) -> np.ndarray:
        a = self.acceptance()
        return np.array([a[i, i + 1] for i in range(self.n - 1)])


class ReplicaExchange:
    """Temperature exchange over `replicas`, an object with

        potentials() -> (R_local,) potential energies [kJ/mol] of its systems (last step),
        set_temperatures(temps (R_local,)), scale_momenta(factors (R_local,)),

    (RigidReplicas wraps a RigidMD batch).  Globally the R = sum of R_local systems of all ranks
    are numbered rank-major; state k of the ladder is held by system `system_at[k]`.

    group: a torch.distributed process group (None: one process).  Every rank must call exchange()
    at the same steps; the uniforms come from one generator seeded identically on all ranks.
    """

    def __init__(self, replicas, temperatures, seed: int = 0, group=None) -> None:
        self.replicas = replicas
        self.temperatures = np.asarray(temperatures, float)
        self.group = group
        self.n = len(self.temperatures)
        self.rng = np.random.default_rng(seed)
        counts = self._allgather(np.array([len(replicas.potentials())], float)).astype(int)
        self.offsets = np.concatenate([[0], np.cumsum(counts)])
        self.rank = 0 if group is None else _dist().get_rank(group)
        if self.offsets[-1] != self.n:
            raise ValueError(f"{self.offsets[-1]} systems for {self.n} temperatures")
        self.system_at = np.arange(self.n)  # state -> global system
        self.stats = ExchangeStatistics(self.n)
        self._apply(np.ones(self.n))

    def _allgather(self, x: np.ndarray) -> np.ndarray:
        if self.group is None:
            return np.asarray(x, float)
        import torch

        dist = _dist()
        t = torch.tensor(np.asarray(x, float), dtype=torch.float64)
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(dist.get_world_size(self.group))]
        dist.all_gather(sizes, torch.tensor([t.numel()], dtype=torch.int64), group=self.group)
        m = int(max(s.item() for s in sizes))
        pad = torch.zeros(m, dtype=torch.float64)
        pad[: t.numel()] = t
        out = [torch.zeros(m, dtype=torch.float64) for _ in sizes]
        dist.all_gather(out, pad, group=self.group)
        return np.concatenate([o[: int(s.item())].numpy() for o, s in zip(out, sizes)])

    def temperature_of_system(self) -> np.ndarray:
        """Temperature [K] of every global system."""
        t = np.empty(self.n)
        t[self.system_at] = self.temperatures
        return t

    def _apply(self, factors_global: np.ndarray) -> None:
        lo, hi = self.offsets[self.rank], self.offsets[self.rank + 1]
        self.replicas.set_temperatures(self.temperature_of_system()[lo:hi])
        f = factors_global[lo:hi]
        if np.any(f != 1.0):
            self.replicas.scale_momenta(f)

    def exchange(self) -> np.ndarray:
        """One round of the even or odd pairs; returns the accepted flags per pair."""
        U_sys = self._allgather(np.asarray(self.replicas.potentials(), float))
        U_state = U_sys[self.system_at]  # potential of the configuration now in each state
        pairs = exchange_pairs(self.n, self.stats.n_exchanges)
        uniforms = self.rng.random(len(pairs))
        u = temperature_reduced_energies(self.temperatures, U_state)
        accepted, src = metropolis(u, pairs, uniforms)
        old_t = self.temperature_of_system()
        self.system_at = self.system_at[src]
        self.stats.record(pairs, accepted, src)
        new_t = self.temperature_of_system()
        self._apply(np.sqrt(new_t / old_t))
        return accepted


class RigidReplicas:
    """Replicas that are systems of a RigidMD batch (by default all of them; `systems` selects a
    subset, e.g. the replicas beside other boxes of the same launch) for ReplicaExchange."""

    def __init__(self, md, systems=None) -> None:
        self.md = md
        self.systems = np.arange(md.ff.nsys) if systems is None else np.asarray(systems, int)

    def potentials(self) -> np.ndarray:
        self.md.stream.synchronize()
        return self.md.result.energy["total"].cpu().numpy()[self.systems]

    def set_temperatures(self, temps) -> None:
        t = np.array(self.md.temps, float)
        t[self.systems] = temps
        self.md.set_temperatures(t)

    def scale_momenta(self, factors) -> None:
        f = np.ones(self.md.ff.nsys)
        f[self.systems] = factors
        self.md.scale_momenta(f)


def _dist():
    import torch.distributed as dist

    return dist
