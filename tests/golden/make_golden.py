"""Write tests/golden/*.npz from the reference's own regression golden files and example frame.

Run once in a container where a checkout of pGM-JAX is available (it is not needed afterwards);
the checkout's root is the one required argument:

    python tests/golden/make_golden.py <path of the pGM-JAX checkout>

ff_small_box.npz -- from tests/regression/golden/ff_small_box.npz of pGM-JAX (case `ff_small_box`,
tests/regression/regression_cases.py:240-276): the MD force field on the 114-atom triclinic
water/methanol box of pgm_jax/models/toy.py:143 small_box(0), cutoff 0.6 nm, skin 0.05, Ewald 6.0/nm,
PME 32^3 order 6, LJ tail, tol 1e-10, max_iter 500, recorded in float64 and in mixed precision.
The inputs (positions, box) are regenerated here by pgm_jax_b200.systems.small_box(0) from the same
numpy seed and stored next to the outputs, so that the tests need neither the reference nor numpy's
generator to stay stable.

iel_point.npz -- from tests/regression/golden/iel_point.npz (case `iel_point`,
regression_cases.py:334-352): the iEL/0-SCF force field (block preconditioner) at small_box(1),
cutoff 0.6 nm, Ewald 6.0/nm, PME 48^3 order 8, float64, tol 1e-10, max_iter 200, from a fresh
solver state (the warm-up solve to tol); inputs regenerated by small_box(1) as above.

ff_pgm3p25_512.npz -- from tests/regression/golden/ff_pgm3p25_512.npz of pGM-JAX (case
`ff_pgm3p25_512`, regression_cases.py:291-307): 512 pGM3P-25 waters of examples/water512, default
MDSettings (cutoff 0.9 nm, Ewald 4.0/nm, order 6, spacing 0.08 nm -> 30^3 on this box, tol 1e-5,
mu4) in float64 and mixed precision.  The frame is examples/water512/pgm3p25_512.rst7 (an Amber
NetCDF restart: coordinates and velocities in Angstrom and Angstrom/ps -- velocities scaled by the
variable's scale_factor as pgm_jax/md/io.py:54-70 reads them -- and a truncated-octahedron cell,
27.201 A, 109.47 deg), turned into the lower-triangular box of pgm_jax/md/box.py:291-314
(box_from_cell) and nm as the regression case does.  The velocities are stored for the 10-step NVE
install check of tests/test_water512.py (step-10 Epot -2114884.256504 kJ/mol, T 291.356783 K).

pmemd_pbc_512.npz -- the independent pmemd-pgm (Amber) single point on the same frame, as the
reference keeps it in data/validation/amber_ref/pmemd_pbc (mdin: cut 10 A, ew_coeff 0.38 / A, PME
72^3 order 8, vdwmeth 0, dipole_scf_tol 1e-9): step-0 EELEC and VDWAALS of mdout [kcal/mol], the
forces of mdfrc [kcal/mol/A, stored as FP32 by pmemd], and the induced dipoles of the last CG
iterate cpu_cg_iter_041.dat [e A].  Amber's pGM uses Tinker's Coulomb constant; the comparison
scales the electrostatic energy and forces by 332.05382 kcal/mol A / (138.935458 kJ/mol nm / 4.184
* 10) as scripts/validation/validate_amber.py does.
"""

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pgm_jax_b200.systems import small_box  # noqa: E402

KEYS = ("energy.elec", "energy.vdw", "energy.total", "forces", "mu", "iterations", "residual", "strain")


def box_from_cell(lengths, angles) -> np.ndarray:
    """Lattice vectors as rows, a along x, b in the xy plane (the Amber / PDB convention)."""
    a, b, c = (float(x) for x in lengths)
    al, be, ga = np.radians(np.asarray(angles, float))
    cx = c * np.cos(be)
    cy = c * (np.cos(al) - np.cos(be) * np.cos(ga)) / np.sin(ga)
    return np.array([[a, 0.0, 0.0], [b * np.cos(ga), b * np.sin(ga), 0.0], [cx, cy, np.sqrt(c * c - cx * cx - cy * cy)]])


def water512_frame(ref: str):
    """(positions [nm], velocities [nm/ps], box [nm]) of examples/water512/pgm3p25_512.rst7."""
    from scipy.io import netcdf_file

    f = netcdf_file(os.path.join(ref, "examples", "water512", "pgm3p25_512.rst7"), "r", mmap=False)
    v = f.variables
    xyz = np.array(v["coordinates"][:], float).reshape(-1, 3)
    vel = np.array(v["velocities"][:], float).reshape(-1, 3) * float(getattr(v["velocities"], "scale_factor", 20.455))
    H = box_from_cell(np.array(v["cell_lengths"][:], float), np.array(v["cell_angles"][:], float))
    return xyz * 0.1, vel * 0.1, H * 0.1


def main(ref: str) -> None:
    gdir = os.path.join(ref, "tests", "regression", "golden")
    g = np.load(os.path.join(gdir, "ff_small_box.npz"))
    _, pos, H = small_box(0)
    out = {"pos": pos, "box": H}
    for tag in ("double", "mixed"):
        for k in KEYS:
            out[f"{tag}.{k}"] = g[f"{tag}.{k}"]
    np.savez_compressed(os.path.join(HERE, "ff_small_box.npz"), **out)
    print("wrote", os.path.join(HERE, "ff_small_box.npz"), sorted(out))

    g = np.load(os.path.join(gdir, "iel_point.npz"))
    _, pos, H = small_box(1)
    out = {"pos": pos, "box": H}
    for k in KEYS:
        out[f"sp.{k}"] = g[f"sp.{k}"]
    np.savez_compressed(os.path.join(HERE, "iel_point.npz"), **out)
    print("wrote", os.path.join(HERE, "iel_point.npz"), sorted(out))

    g = np.load(os.path.join(gdir, "ff_pgm3p25_512.npz"))
    pos, vel, H = water512_frame(ref)
    out = {"pos": pos, "vel": vel, "box": H}
    for tag in ("double", "mixed"):
        for k in KEYS:
            out[f"{tag}.{k}"] = g[f"{tag}.{k}"]
    np.savez_compressed(os.path.join(HERE, "ff_pgm3p25_512.npz"), **out)
    print("wrote", os.path.join(HERE, "ff_pgm3p25_512.npz"), sorted(out))

    out = pmemd_pbc(ref)
    np.savez_compressed(os.path.join(HERE, "pmemd_pbc_512.npz"), **out)
    print("wrote", os.path.join(HERE, "pmemd_pbc_512.npz"), sorted(out))


def pmemd_pbc(ref: str) -> dict:
    """Step-0 energies, forces and induced dipoles of the reference's stored pmemd-pgm run."""
    from scipy.io import netcdf_file

    d = os.path.join(ref, "data", "validation", "amber_ref", "pmemd_pbc")
    txt = open(os.path.join(d, "mdout")).read()
    blk = txt[txt.index("NSTEP =        0"):]
    get = lambda k: float(re.search(rf"{k}\s*=\s*(-?\d+\.\d+)", blk).group(1))  # noqa: E731
    f = netcdf_file(os.path.join(d, "mdfrc"), "r", mmap=False)
    forces = np.array(f.variables["forces"][:], float)[0]
    f.close()
    mu = np.loadtxt(os.path.join(d, "cpu_cg_iter_041.dat"), comments="#")[:, 1:4]
    return {"eelec_kcal": get("EELEC"), "vdw_kcal": get("VDWAALS"), "forces_kcal_A": forces, "mu_e_A": mu}


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
