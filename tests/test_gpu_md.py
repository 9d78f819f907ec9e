"""Rigid-body MD on the engine: captured CUDA-graph steps equal direct steps; NVE conserves energy."""

import numpy as np
import pytest
from conftest import SMALL_BOX_SETTINGS

pytestmark = pytest.mark.gpu


def make_md(system, pos, H, prec="double", gamma=0.0, dt=0.5, **kw):
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD

    st = dict(SMALL_BOX_SETTINGS, dipole_tol=1e-9, max_iter=200)
    st.update(kw)
    ff = PGMForceField(system, H, MDSettings(precision=prec, **st))
    return RigidMD(ff, pos, H, temperature=300.0, dt_fs=dt, gamma_ps=gamma, seed=3)


@pytest.mark.parametrize("gamma,niter", [(0.0, 0), (5.0, 0), (5.0, 2)])
def test_graph_replay_equals_direct_steps(small_box_system, gamma, niter):
    """The captured step (CG as a device-side while loop, row field beside the FFTs; with niter > 0
    the local preconditioner's chain inside the loop) is the direct step."""
    s, pos, H = small_box_system
    a = make_md(s, pos, H, gamma=gamma, local_niter=niter)
    b = make_md(s, pos, H, gamma=gamma, local_niter=niter)
    for _ in range(4):
        a.step()
    b.capture()
    b.run(4)
    ea, eb = a.energy(), b.energy()
    assert abs(ea["total"][0] - eb["total"][0]) <= 1e-9 * abs(ea["total"][0])
    assert np.abs(a.pos.cpu().numpy() - b.pos.cpu().numpy()).max() < 1e-10
    assert int(a.ff._iters[0]) == int(b.ff._iters[0])


def test_nve_conserves_energy(small_box_system):
    """40 NVE steps of 0.5 fs: kinetic + potential energy drifts by < 0.5 % of the kinetic energy."""
    s, pos, H = small_box_system
    md = make_md(s, pos, H, dt=0.5, peek=0.0)
    e0 = md.energy()
    tot0 = e0["total"][0] + e0["kinetic"][0]
    md.capture()
    for _ in range(4):
        md.run(10)
        e = md.energy()
        tot = e["total"][0] + e["kinetic"][0]
        assert abs(tot - tot0) < 5e-3 * e0["kinetic"][0], (tot, tot0, e0["kinetic"][0])


def test_langevin_reaches_temperature():
    """A Langevin run (gamma 20 / ps) of 64 rigid waters holds the temperature near its target."""
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(4, 1.25, seed=2)
    ff = PGMForceField(s, H, MDSettings(precision="mixed", cutoff=0.6, ewald_beta=6.0, pme_grid=(24, 24, 24),
                                        dipole_tol=1e-6))
    md = RigidMD(ff, pos, H, temperature=300.0, dt_fs=1.0, gamma_ps=20.0, seed=5)
    md.capture()
    temps = []
    for _ in range(30):
        md.run(10)
        temps.append(md.temperature()[0])
    assert 240.0 < np.mean(temps[10:]) < 360.0, temps


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_water512_install_check(pgm3p25_512_system, golden_pgm3p25_512, prec):
    """The reference's install check (tests/test_water512.py): 10 NVE steps of 1 fs from
    examples/water512 (512 pGM3P-25 waters with the file's velocities) at the run_md defaults
    (cutoff 0.9 nm, Ewald 4.0 / nm, PME 48^3 order 8, LJ tail, tol 1e-5, mu4).  Step-10 potential
    energy -2114884.256504 kJ/mol within 1e-9 (FP64) or 1e-6 (mixed), temperature 291.356783 K
    within 1e-6 (1e-5 mixed), total energy between steps 5 and 10 within 0.5 kJ/mol."""
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD

    g = golden_pgm3p25_512
    st = dict(cutoff=0.9, ewald_beta=4.0, pme_grid=(48, 48, 48), pme_order=8, lj_lrc=True, dipole_tol=1e-5, max_iter=50)
    ff = PGMForceField(pgm3p25_512_system, g["box"], MDSettings(precision=prec, **st))
    md = RigidMD(ff, g["pos"], g["box"], temperature=298.0, dt_fs=1.0, gamma_ps=0.0, velocities=g["vel"])
    etot = []
    for _ in range(10):
        md.step()
        e = md.energy()
        etot.append(e["total"][0] + e["kinetic"][0])
    epot, T = md.energy()["total"][0], md.temperature()[0]
    rtol_e, rtol_t = (1e-9, 1e-6) if prec == "double" else (1e-6, 1e-5)
    assert abs(epot - -2114884.256504) <= rtol_e * 2114884.256504, epot
    assert abs(T - 291.356783) <= rtol_t * 291.356783, T
    assert abs(etot[9] - etot[4]) < 0.5
    assert int(md.result.status[0]) == 0


def test_c1_nve_trajectory_matches_oracle():
    """The FP64 configuration of the benchmarks (512 rigid pGM3P-25 waters on the seeded jittered
    8x8x8 lattice, 2.483 nm box, cutoff 0.9 nm, Ewald 4.0 / nm, PME 48^3 order 6, CG 1e-8, Maxwell
    velocities at 298 K, NVE, dt 1 fs, 10 steps) against the NumPy NO_SQUISH restatement driven by
    the FP64 oracle's forces: potential energy every step within 1e-9 relative, final positions
    within 1e-9 nm."""
    import sys

    sys.path.insert(0, __import__("os").path.join(__import__("os").path.dirname(__file__), "..", "oracle"))
    import oracle as O
    from rigid_oracle import RigidNVE

    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(8, 2.483, seed=0)
    rng = np.random.default_rng(11)
    kT = 0.0083144626181532 * 298.0
    vel = rng.normal(size=(s.n, 3)) * np.sqrt(kT / np.asarray(s.masses, float))[:, None]
    st = dict(cutoff=0.9, ewald_beta=4.0, pme_grid=(48, 48, 48), pme_order=6, lj_lrc=True, dipole_tol=1e-8, max_iter=100)
    ff = PGMForceField(s, H, MDSettings(precision="double", **st))
    md = RigidMD(ff, pos, H, temperature=298.0, dt_fs=1.0, gamma_ps=0.0, velocities=vel)
    o = O.Oracle(s, st)
    state = {"ind": o.init_induction()}

    def forces(x):
        r = o.compute(x, H, state["ind"])
        state["ind"] = r["induction"]
        return r["forces"], r["energy"]["total"]

    ref = RigidNVE(s, pos, H, vel, forces)
    for step in range(10):
        md.step()
        ref.step(0.001)
        e = float(md.energy()["total"][0])
        assert abs(e - ref.epot) <= 1e-9 * abs(ref.epot), (step, e, ref.epot)
    assert np.abs(md.pos.cpu().numpy() - ref.positions()).max() <= 1e-9
    assert int(md.result.status[0]) == 0
