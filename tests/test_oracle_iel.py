"""The oracle's extended-Lagrangian dipoles (iEL/0-SCF, iEL/SCF; pgm_jax/md/forcefield.py:1452-1650,
2011-2045, 2294-2360) against the reference's iel_point golden and the physics of the shadow
potential (no GPU)."""

import numpy as np
import pytest
from conftest import IEL_POINT_SETTINGS

import oracle as O


def test_iel_point_matches_reference_golden(golden_iel_point):
    """A fresh state takes the warm-up solve to tol (regression case iel_point, block preconditioner)."""
    from pgm_jax_b200.systems import small_box

    g = golden_iel_point
    s, pos, H = small_box(1)
    assert np.array_equal(pos, g["pos"]) and np.array_equal(H, g["box"])
    r = O.Oracle(s, IEL_POINT_SETTINGS).compute(pos, H)
    for k in ("elec", "vdw", "total"):
        ref = float(g[f"sp.energy.{k}"])
        assert abs(r["energy"][k] - ref) <= 1e-10 * abs(ref), (k, r["energy"][k], ref)
    assert r["iterations"] == int(g["sp.iterations"])
    assert np.abs(r["forces"] - g["sp.forces"]).max() <= 1e-8 * np.abs(g["sp.forces"]).max()
    assert np.abs(r["mu"] - g["sp.mu"]).max() <= 1e-9 * np.abs(g["sp.mu"]).max()
    assert np.abs(r["virial"] - g["sp.strain"]).max() <= 1e-7 * np.abs(g["sp.strain"]).max()


def _walk(o, s, pos, H, steps, seed=0):
    """`steps` steps along a straight drift (every atom 0.3 nm/ps Gaussian, 1 fs): the warm-up, then
    extended steps; returns the positions and state before the last step and the last result."""
    v = np.random.default_rng(seed).normal(scale=0.3, size=pos.shape)
    ind, x = o.init_induction(), pos.copy()
    r = None
    for _ in range(steps):
        x = x + v * 1e-3
        prev = ind
        r = o.compute(x, H, ind)
        ind = r["induction"]
    return x, prev, r, ind


@pytest.mark.parametrize("precond", ["block", "jacobi"])
def test_0scf_steps_take_no_cg_and_forces_are_the_shadow_gradient(small_box_system, precond):
    """After the max(K, 2) + 1 warm-up steps the 0-SCF step needs no CG iteration, and its forces are
    the exact gradient of the shadow energy U~(R, x) at fixed auxiliary dipoles x (central
    differences, Richardson-extrapolated, 1e-7 relative)."""
    s, pos, H = small_box_system
    o = O.Oracle(s, dict(IEL_POINT_SETTINGS, pme_grid=(32, 32, 32), pme_order=6, dipole_tol=1e-8, iel_precond=precond))
    x, ind_prev, r, _ = _walk(o, s, pos, H, 11)
    assert r["iterations"] == 0 and 0 < r["residual"] < 1e-2
    for a, c in [(0, 0), (5, 1), (40, 2), (77, 0)]:
        def fd(h):
            d = np.zeros_like(x)
            d[a, c] = h
            return -(o.compute(x + d, H, ind_prev)["energy"]["total"] - o.compute(x - d, H, ind_prev)["energy"]["total"]) / (2 * h)

        ric = (4 * fd(1e-5) - fd(2e-5)) / 3
        assert abs(ric - r["forces"][a, c]) <= 1e-7 * max(1.0, abs(ric)), (a, c, ric, r["forces"][a, c])


def test_0scf_shadow_energy_is_below_the_converged_energy(small_box_system):
    """U~(R, x) = U(R, x) - sum alpha |r|^2 / 2 (Jacobi) differs from the converged U*(R) by a
    second-order amount, and the fixed-dipole forces (shadow off) differ from the shadow forces by a
    second-order amount, at the same dipoles."""
    s, pos, H = small_box_system
    st = dict(IEL_POINT_SETTINGS, pme_grid=(32, 32, 32), pme_order=6, dipole_tol=1e-8, iel_precond="jacobi")
    x, ind_prev, r, _ = _walk(O.Oracle(s, st), s, pos, H, 11)
    conv = O.Oracle(s, dict(st, iel="none", dipole_tol=1e-12, max_iter=500)).compute(x, H)
    gap = conv["energy"]["total"] - r["energy"]["total"]
    assert abs(gap) < 1e-4 * abs(conv["energy"]["total"])
    off = O.Oracle(s, dict(st, iel_shadow=False)).compute(x, H, ind_prev)
    diff = np.abs(off["forces"] - r["forces"]).max()
    assert 0 < diff < 1e-4 * np.abs(r["forces"]).max()  # second order in delta
    assert np.array_equal(off["mu"], r["mu"])


def test_iel_scf_runs_the_set_iterations(small_box_system):
    """iEL/SCF: iel_iter CG iterations from x per extended step (tol 0: exactly that many)."""
    s, pos, H = small_box_system
    o = O.Oracle(s, dict(IEL_POINT_SETTINGS, pme_grid=(32, 32, 32), pme_order=6, dipole_tol=1e-8, iel="scf", iel_iter=2))
    _, _, r, ind = _walk(o, s, pos, H, 11)
    assert r["iterations"] == 2 and r["residual"] < 1e-2 and ind["count"] == 11


def test_auxiliary_dipoles_follow_the_dissipative_verlet_recurrence(small_box_system):
    """x_{n+1} = 2 x_n - x_{n-1} + kappa (mu_n - x_n) + a sum_k c_k x_{n-k} with the order-7 table
    (kappa 1.86, a 0.0016, c = -36, 99, -88, 11, 32, -25, 8, -1)."""
    s, pos, H = small_box_system
    o = O.Oracle(s, dict(IEL_POINT_SETTINGS, pme_grid=(32, 32, 32), pme_order=6, dipole_tol=1e-8))
    x, ind_prev, r, ind = _walk(o, s, pos, H, 12)
    X = ind_prev["xl"]
    c = [-36, 99, -88, 11, 32, -25, 8, -1]
    want = 2 * X[0] - X[1] + 1.86 * (r["mu"] - X[0]) + 0.0016 * sum(ck * X[k] for k, ck in enumerate(c))
    assert np.abs(ind["xl"][0] - want).max() <= 1e-14 * np.abs(want).max()
    assert np.array_equal(ind["xl"][1:], X[:-1]) and X.shape[0] == 9
