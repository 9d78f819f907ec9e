"""Extended-Lagrangian induced dipoles on the GPU (iEL/0-SCF, iEL/SCF; pgm_jax/md/forcefield.py:
1452-1650) against the oracle and the reference's iel_point golden.

Tolerances as the other parity tests: FP64 engine to ~1e-9 of the oracle, mixed precision 1e-6 in
energy and 1e-5 RMS in forces and dipoles."""

import numpy as np
import pytest
from conftest import IEL_POINT_SETTINGS

pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402


def rms_rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b**2)))


def _ff(system, H, prec, **st):
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField

    return PGMForceField(system, H, MDSettings(precision=prec, **st))


def test_iel_point_matches_reference_golden(golden_iel_point):
    from pgm_jax_b200.systems import small_box

    g = golden_iel_point
    s, pos, H = small_box(1)
    ff = _ff(s, H, "double", **IEL_POINT_SETTINGS)
    r = ff.compute(pos, H, None, ff.init_induction())
    assert int(r.status[0]) == 0
    for k in ("elec", "vdw", "total"):
        ref = float(g[f"sp.energy.{k}"])
        assert abs(float(r.energy[k][0]) - ref) <= 1e-9 * abs(ref), (k, float(r.energy[k][0]), ref)
    assert int(r.iterations[0]) == int(g["sp.iterations"])
    assert np.abs(r.forces.cpu().numpy() - g["sp.forces"]).max() <= 1e-8 * np.abs(g["sp.forces"]).max()
    assert np.abs(r.virial[0].cpu().numpy() - g["sp.strain"]).max() <= 1e-7 * np.abs(g["sp.strain"]).max()


@pytest.mark.parametrize("prec", ["double", "mixed"])
@pytest.mark.parametrize("scheme", [dict(iel="0scf", iel_precond="block"), dict(iel="0scf", iel_precond="jacobi"),
                                    dict(iel="0scf", iel_precond="jacobi", iel_omega=0.8, iel_order=5),
                                    dict(iel="scf", iel_iter=2), dict(iel="0scf", iel_shadow=False)])
def test_iel_steps_match_oracle(small_box_system, prec, scheme):
    """12 steps along a smooth drift (the 8 warm-up solves, then extended steps): energies,
    forces, dipoles, the auxiliary dipoles and CG iterations as the oracle's, step by step."""
    s, pos, H = small_box_system
    st = dict(IEL_POINT_SETTINGS, pme_grid=(32, 32, 32), pme_order=6, dipole_tol=1e-8, **scheme)
    o = O.Oracle(s, st)
    ff = _ff(s, H, prec, **st)
    ind_o, ind_g = o.init_induction(), ff.init_induction()
    v = np.random.default_rng(0).normal(scale=0.3, size=pos.shape)
    x = pos.copy()
    tol_e, tol_f = (1e-9, 1e-8) if prec == "double" else (1e-6, 1e-5)
    for step in range(12):
        x = x + v * 1e-3
        ro = o.compute(x, H, ind_o)
        ind_o = ro["induction"]
        rg = ff.compute(x, H, None, ind_g)
        ind_g = rg.induction
        e = float(rg.energy["total"][0])
        assert abs(e - ro["energy"]["total"]) <= tol_e * abs(ro["energy"]["total"]), (step, e, ro["energy"]["total"])
        assert rms_rel(rg.forces.cpu().numpy(), ro["forces"]) <= tol_f, step
        assert rms_rel(ind_g.mu.cpu().numpy(), ro["mu"]) <= tol_f, step
        assert rms_rel(ind_g.xl.cpu().numpy(), ind_o["xl"]) <= tol_f, step
        if prec == "double":
            assert int(rg.iterations[0]) == ro["iterations"], (step, int(rg.iterations[0]), ro["iterations"])
        else:
            assert abs(int(rg.iterations[0]) - ro["iterations"]) <= 1
        assert not int(rg.status[0]) & ~0x2
    assert int(ind_g.count[0]) == 12
    if scheme["iel"] == "0scf":
        assert int(rg.iterations[0]) == 0  # extended 0-SCF steps take no CG iteration


def test_iel_captured_steps_equal_direct_steps(small_box_system):
    """Rigid-body MD with iEL/0-SCF: graph replays (the warm-up solve and the extended step in one
    captured step) equal direct steps; E_kin + the shadow energy is conserved in NVE."""
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD

    s, pos, H = small_box_system
    st = dict(IEL_POINT_SETTINGS, pme_grid=(32, 32, 32), pme_order=6, dipole_tol=1e-8)
    mds = []
    for cap in (False, True):
        ff = PGMForceField(s, H, MDSettings(precision="double", **st))
        md = RigidMD(ff, pos, H, temperature=300.0, dt_fs=0.5, gamma_ps=0.0, seed=3)
        if cap:
            md.capture()
            md.run(20)
        else:
            for _ in range(20):
                md.step()
        mds.append(md)
    a, b = mds
    ea, eb = a.energy(), b.energy()
    assert abs(ea["total"][0] - eb["total"][0]) <= 1e-9 * abs(ea["total"][0])
    assert np.abs(a.pos.cpu().numpy() - b.pos.cpu().numpy()).max() < 1e-10
    tot = []
    for _ in range(8):
        b.run(10)
        e = b.energy()
        tot.append(e["total"][0] + e["kinetic"][0])
    assert max(tot) - min(tot) < 2e-3 * ea["kinetic"][0], tot
