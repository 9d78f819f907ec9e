"""Monte Carlo barostat decision and step-size rules (host arrays; pgm_jax/md/integrate.py:763-817)."""

import numpy as np

from pgm_jax_b200.barostat import KJMOL_NM3_PER_BAR, mc_accept, mc_adapt


def test_acceptance_follows_the_volume_move_weight():
    """w = dE + P dV - M kT ln(V'/V): accepted iff log u < -w / kT, per system; V' <= 0 and a
    non-finite trial energy are rejected."""
    rng = np.random.default_rng(0)
    S = 64
    V = rng.uniform(50, 150, S)
    dV = rng.uniform(-2, 2, S)
    e_old = rng.normal(-1e5, 10, S)
    e_new = e_old + rng.normal(0, 5, S)
    nmol = rng.integers(100, 2000, S)
    kT = rng.uniform(2.0, 3.0, S)
    P = 1.0 * KJMOL_NM3_PER_BAR
    log_u = np.log(rng.uniform(size=S))
    got = mc_accept(e_new, e_old, dV, V, nmol, kT, P, log_u)
    w = (e_new - e_old) + P * dV - nmol * kT * np.log((V + dV) / V)
    assert np.array_equal(got, log_u < -w / kT)
    assert 0 < got.sum() < S
    assert not mc_accept([0.0], [0.0], [-200.0], [100.0], [10], [2.5], P, [-50.0])[0]  # V' < 0
    assert not mc_accept([np.nan], [0.0], [1.0], [100.0], [10], [2.5], P, [-50.0])[0]
    # a compression with no energy change at a large pressure is always accepted
    assert mc_accept([0.0], [0.0], [-1.0], [100.0], [10], [2.5], 1e4 * KJMOL_NM3_PER_BAR, [np.log(0.999)])[0]


def test_step_size_adapts_after_ten_tries():
    dv, t, a = mc_adapt([1.0, 1.0, 1.0, 1.0], [10, 10, 10, 9], [1, 9, 5, 0], [100.0, 100.0, 100.0, 100.0])
    assert np.allclose(dv, [1 / 1.1, 1.1, 1.0, 1.0])
    assert list(t) == [0, 0, 0, 9] and list(a) == [0, 0, 0, 0]
    dv, _, _ = mc_adapt([29.0], [10], [10], [100.0])
    assert dv[0] == 30.0  # at most 0.3 V
    assert abs(KJMOL_NM3_PER_BAR - 0.0602214) < 1e-6
