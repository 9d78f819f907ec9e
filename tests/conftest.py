"""Shared test setup: the `gpu` marker, import paths and the fixtures of the golden box."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# Settings of the reference's regression case ff_small_box (regression_cases.py:253-262)
SMALL_BOX_SETTINGS = dict(
    cutoff=0.6, ewald_beta=6.0, pme_grid=(32, 32, 32), pme_order=6, lj_lrc=True, dipole_tol=1e-10, max_iter=500
)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden_small_box():
    return dict(np.load(os.path.join(GOLDEN, "ff_small_box.npz")))


# Settings of the reference's regression case ff_pgm3p25_512 (regression_cases.py:291-307): the
# MDSettings defaults; the 0.08 nm spacing gives a 30^3 mesh on the 2.72 nm truncated octahedron
PGM3P25_512_SETTINGS = dict(
    cutoff=0.9, ewald_beta=4.0, pme_grid=(30, 30, 30), pme_order=6, lj_lrc=True, dipole_tol=1e-5, max_iter=50
)


@pytest.fixture(scope="session")
def golden_pgm3p25_512():
    return dict(np.load(os.path.join(GOLDEN, "ff_pgm3p25_512.npz")))


@pytest.fixture(scope="session")
def golden_pmemd_pbc_512():
    return dict(np.load(os.path.join(GOLDEN, "pmemd_pbc_512.npz")))


# The pmemd-pgm single point of the same 512-water frame (data/validation/amber_ref/pmemd_pbc/mdin
# of pGM-JAX): cut 10 A, ew_coeff 0.38 / A, PME 72^3 order 8, vdwmeth 0 (no LJ tail), SCF tol 1e-9.
PMEMD_PBC_SETTINGS = dict(cutoff=1.0, ewald_beta=3.8, pme_grid=(72, 72, 72), pme_order=8, lj_lrc=False,
                          dipole_tol=1e-10, max_iter=500)
# Amber's pGM uses Tinker's Coulomb constant: electrostatic energy and forces scale by this ratio
# (scripts/validation/validate_amber.py of pGM-JAX, units.py:31-36).
AMBER_KE_SCALE = (332.05382 * 4.184 / 10.0) / 138.935458


def pmemd_compare(energy_elec_kj, energy_vdw_kj, forces_elec, forces_total, mu_nm, golden):
    """(EELEC relative deviation, VDWAALS deviation [kcal/mol], force RMSD [kcal/mol/A], dipole RMSD
    [e A]) against the stored pmemd-pgm run, from our electrostatic-only and total forces [kJ/mol/nm]."""
    e = energy_elec_kj / 4.184 * AMBER_KE_SCALE
    f = (forces_elec * AMBER_KE_SCALE + (forces_total - forces_elec)) / 41.84
    rms = lambda x: float(np.sqrt(np.mean(x * x)))  # noqa: E731
    return (abs(e - float(golden["eelec_kcal"])) / abs(float(golden["eelec_kcal"])),
            abs(energy_vdw_kj / 4.184 - float(golden["vdw_kcal"])), rms(f - golden["forces_kcal_A"]),
            rms(10.0 * mu_nm - golden["mu_e_A"]))


@pytest.fixture(scope="session")
def pgm3p25_512_system():
    from pgm_jax_b200.systems import System, pgm3p25_water

    return System([pgm3p25_water()] * 512)


@pytest.fixture(scope="session")
def small_box_system():
    from pgm_jax_b200.systems import small_box

    return small_box(0)


# Settings of the reference's regression case iel_point (regression_cases.py:334-352)
IEL_POINT_SETTINGS = dict(
    cutoff=0.6, ewald_beta=6.0, pme_grid=(48, 48, 48), pme_order=8, lj_lrc=True, dipole_tol=1e-10, max_iter=200,
    iel="0scf", iel_precond="block",
)


@pytest.fixture(scope="session")
def golden_iel_point():
    return dict(np.load(os.path.join(GOLDEN, "iel_point.npz")))
