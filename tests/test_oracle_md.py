"""The NumPy restatement of the reference's rigid-body NVE step (oracle/rigid_oracle.py) with the
FP64 oracle's forces reproduces the reference's install check (no GPU).

tests/test_water512.py of pGM-JAX runs `pgm-jax md` for 10 NVE steps of 1 fs from
examples/water512 (512 pGM3P-25 waters, truncated octahedron, with the file's velocities) at the
run_md defaults (scripts/md/run_md.py: cutoff 9 A, Ewald 0.4 / A, PME spacing 0.5 A -> 48^3 here,
order 8, LJ tail, tol 1e-5, mu4) and checks the step-10 potential energy against
-2114884.256504 kJ/mol (1e-9 relative, float64) and the temperature against 291.356783 K (1e-6).
"""

import numpy as np

import oracle as O
from rigid_oracle import RigidNVE

EPOT_REF = -2114884.256504  # kJ/mol, step 10 (tests/test_water512.py:26)
TEMP_REF = 291.356783  # K (tests/test_water512.py:27)
WATER512_MD = dict(cutoff=0.9, ewald_beta=4.0, pme_grid=(48, 48, 48), pme_order=8, lj_lrc=True, dipole_tol=1e-5,
                   max_iter=50)


def test_water512_install_check_on_the_oracle(pgm3p25_512_system, golden_pgm3p25_512):
    g = golden_pgm3p25_512
    o = O.Oracle(pgm3p25_512_system, WATER512_MD)
    state = {"ind": o.init_induction()}

    def forces(x):
        r = o.compute(x, g["box"], state["ind"])
        state["ind"] = r["induction"]
        return r["forces"], r["energy"]["total"]

    md = RigidNVE(pgm3p25_512_system, g["pos"], g["box"], g["vel"], forces)
    e = [md.epot + md.kinetic()]
    for _ in range(10):
        md.step(0.001)
        e.append(md.epot + md.kinetic())
    assert abs(md.epot - EPOT_REF) <= 1e-9 * abs(EPOT_REF), md.epot
    assert abs(md.temperature() - TEMP_REF) <= 1e-6 * TEMP_REF, md.temperature()
    assert abs(e[10] - e[5]) < 0.5  # the reference's conservation check between the two log rows


def test_no_squish_rotations_keep_unit_quaternions_and_angular_momentum(pgm3p25_512_system, golden_pgm3p25_512):
    """The free rotor alone conserves |q| = 1, q . p and every body's |L| (each exact rotation about
    a principal axis turns L about that axis); its kinetic energy only to the splitting's order."""
    from rigid_oracle import perm

    g = golden_pgm3p25_512
    md = RigidNVE(pgm3p25_512_system, g["pos"], g["box"], g["vel"], lambda x: (np.zeros_like(x), 0.0))

    def L2():
        return sum((0.5 * np.sum(perm(k, md.q) * md.p, 1)) ** 2 for k in (1, 2, 3))

    k0, qp0, l0 = md.kinetic(), np.sum(md.q * md.p, 1), L2()
    for _ in range(50):
        md.free_rotor(0.002)
    assert np.abs(np.linalg.norm(md.q, axis=1) - 1).max() < 1e-13
    assert np.abs(np.sum(md.q * md.p, 1) - qp0).max() < 1e-12
    assert np.abs(L2() - l0).max() < 1e-12 * l0.max()
    assert abs(md.kinetic() - k0) < 1e-4 * k0
