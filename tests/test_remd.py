"""Replica exchange: the ladder, the pairing and the Metropolis criterion (as pgm_jax/md/remd.py
defines them), the exchange chain against the exact stationary distribution over permutations,
the bookkeeping of temperatures and momentum factors, and the same decisions from two gloo ranks
that each hold half of the replicas."""

import itertools
import os
import socket

import numpy as np
import pytest

from pgm_jax_b200.remd import (
    KB,
    ReplicaExchange,
    exchange_pairs,
    geometric_ladder,
    metropolis,
    temperature_reduced_energies,
)


class FixedEnergies:
    """Configurations (one per system) with fixed potential energies and no dynamics."""

    def __init__(self, energies):
        self.E = np.asarray(energies, float)
        self.temps = None
        self.factors = []

    def potentials(self):
        return self.E.copy()

    def set_temperatures(self, temps):
        self.temps = np.asarray(temps, float).copy()

    def scale_momenta(self, factors):
        self.factors.append(np.asarray(factors, float).copy())


def test_ladder_pairs_and_criterion():
    T = geometric_ladder(300.0, 450.0, 5)
    assert np.isclose(T[0], 300.0) and np.isclose(T[-1], 450.0) and np.allclose(T[1:] / T[:-1], 1.5**0.25)
    assert exchange_pairs(5, 0) == [(0, 1), (2, 3)] and exchange_pairs(5, 1) == [(1, 2), (3, 4)]
    assert exchange_pairs(4, 3) == [(1, 2)]
    U = np.array([-100.0, -90.0])
    u = temperature_reduced_energies([300.0, 330.0], U)
    p = np.exp(-(1.0 / (KB * 300.0) - 1.0 / (KB * 330.0)) * (U[1] - U[0]))
    assert 0.0 < p < 1.0
    assert metropolis(u, [(0, 1)], [p * 0.999])[0][0] and not metropolis(u, [(0, 1)], [p * 1.001])[0][0]
    acc, src = metropolis(temperature_reduced_energies([300.0, 330.0], U[::-1]), [(0, 1)], [0.9999])
    assert acc[0] and list(src) == [1, 0]  # downhill: always
    V, P = np.array([30.0, 31.0]), 0.0602214
    assert np.allclose(temperature_reduced_energies([300.0, 330.0], U, V, P),
                       temperature_reduced_energies([300.0, 330.0], U + P * V))
    with pytest.raises(ValueError):
        metropolis(u, [(0, 1), (1, 0)], [0.5, 0.5])
    with pytest.raises(ValueError):
        geometric_ladder(300.0, 200.0, 4)
    with pytest.raises(FloatingPointError):
        metropolis(np.array([[0.0, np.inf], [0.0, 0.0]]), [(0, 1)], [0.5])


def test_exchange_chain_samples_the_permutation_distribution():
    """Exchanges only: the states' configurations follow pi(sigma) ~ exp(-sum_k beta_k E_sigma(k))
    and each pair's acceptance is E_pi[min(1, e^-Delta)]; temperatures and momentum factors follow
    the configurations."""
    T = geometric_ladder(300.0, 420.0, 4)
    E = np.array([0.0, 25.0, 60.0, 110.0])
    reps = FixedEnergies(E)
    rex = ReplicaExchange(reps, T, seed=3)
    perms = list(itertools.permutations(range(4)))
    index = {p: i for i, p in enumerate(perms)}
    counts = np.zeros(len(perms))
    n = 60000
    for _ in range(n):
        before = rex.temperature_of_system()
        nf = len(reps.factors)
        rex.exchange()
        after = rex.temperature_of_system()
        assert np.allclose(reps.temps, after)
        if not np.array_equal(before, after):
            assert len(reps.factors) == nf + 1 and np.allclose(reps.factors[-1], np.sqrt(after / before))
        counts[index[tuple(rex.system_at)]] += 1
    beta = 1.0 / (KB * T)
    w = np.array([np.exp(-np.sum(beta * E[list(p)])) for p in perms])
    w /= w.sum()
    assert 0.5 * np.abs(counts / n - w).sum() < 0.01
    acc = rex.stats.neighbour_acceptance()
    for i in range(3):
        exact = sum(wp * min(1.0, np.exp(-(beta[i] - beta[i + 1]) * (E[p[i + 1]] - E[p[i]]))) for p, wp in zip(perms, w))
        assert abs(acc[i] - exact) < 0.01, (i, acc[i], exact)
        assert rex.stats.attempts[i, i + 1] == n // 2
    assert np.array_equal(rex.stats.replica, rex.system_at)
    assert rex.stats.round_trips.sum() > 100 and np.all(rex.stats.transits >= 2 * rex.stats.round_trips)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, E, T, n, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        k = len(E) // world
        reps = FixedEnergies(E[rank * k:(rank + 1) * k])
        rex = ReplicaExchange(reps, T, seed=7, group=dist.group.WORLD)
        hist = []
        for _ in range(n):
            rex.exchange()
            hist.append(rex.system_at.copy())
        np.save(os.path.join(out, f"r{rank}.npy"), np.array(hist))
        np.save(os.path.join(out, f"t{rank}.npy"), reps.temps)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_single_process_decisions(tmp_path):
    """Four replicas on two ranks (an all-gather of the energies per exchange) walk exactly as the
    same four in one process; each rank's systems get the temperatures of their states."""
    import torch.multiprocessing as mp

    T = geometric_ladder(280.0, 400.0, 4)
    E = np.array([10.0, -5.0, 30.0, 22.0])
    n = 300
    mp.start_processes(_rank, args=(2, _free_port(), E, T, n, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    single = ReplicaExchange(FixedEnergies(E), T, seed=7)
    ref = []
    for _ in range(n):
        single.exchange()
        ref.append(single.system_at.copy())
    ref = np.array(ref)
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"r{r}.npy"), ref)
    temps = np.concatenate([np.load(tmp_path / f"t{r}.npy") for r in range(2)])
    assert np.allclose(temps, single.temperature_of_system())
