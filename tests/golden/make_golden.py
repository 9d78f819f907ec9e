"""Write tests/golden/*.npz from the reference's own regression golden files.

Run in a container where the reference is mounted (it is not needed afterwards):

    python tests/golden/make_golden.py /root/reference

Source: tests/regression/golden/ff_small_box.npz of pGM-JAX (case `ff_small_box`,
tests/regression/regression_cases.py:240-276): the MD force field on the 114-atom triclinic
water/methanol box of pgm_jax/models/toy.py:143 small_box(0), cutoff 0.6 nm, skin 0.05, Ewald 6.0/nm,
PME 32^3 order 6, LJ tail, tol 1e-10, max_iter 500, recorded in float64 and in mixed precision.
The inputs (positions, box) are regenerated here by pgm_jax_b200.systems.small_box(0) from the same
numpy seed and stored next to the outputs, so that the tests need neither the reference nor numpy's
generator to stay stable.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pgm_jax_b200.systems import small_box  # noqa: E402


def main(ref: str) -> None:
    g = np.load(os.path.join(ref, "tests", "regression", "golden", "ff_small_box.npz"))
    _, pos, H = small_box(0)
    out = {"pos": pos, "box": H}
    for tag in ("double", "mixed"):
        for k in ("energy.elec", "energy.vdw", "energy.total", "forces", "mu", "iterations", "residual", "strain"):
            out[f"{tag}.{k}"] = g[f"{tag}.{k}"]
    np.savez_compressed(os.path.join(HERE, "ff_small_box.npz"), **out)
    print("wrote", os.path.join(HERE, "ff_small_box.npz"), sorted(out))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
