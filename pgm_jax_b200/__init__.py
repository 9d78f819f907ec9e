"""B200-native (sm_100a) per-step pGM polarizable electrostatics with the call surface of pGM-JAX's
PGMForceField (pgm_jax/md/forcefield.py): pair rows, smooth PME and the induced-dipole CG solve in
hand-written CUDA behind a C ABI (include/pgm_b200.h)."""

from .systems import Molecule, System, grid_size, pgm3p25_water, small_box, water_box  # noqa: F401

__all__ = ["Molecule", "System", "grid_size", "pgm3p25_water", "small_box", "water_box", "PGMForceField", "MDSettings"]


def __getattr__(name):
    if name in ("PGMForceField", "MDSettings", "InductionState", "Result"):
        from . import forcefield

        return getattr(forcefield, name)
    raise AttributeError(name)
