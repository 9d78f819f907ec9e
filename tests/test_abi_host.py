"""No-GPU checks: the C ABI library exports every declared symbol, and the host-side logic."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            names += re.findall(r"^\s*(?:PgmStatus|int|long long|const char \*)\s*\**\s*(pgm_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_builds_and_exports_every_declared_symbol():
    from pgm_jax_b200 import _lib, build

    build.build()
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.EXPORTS)


def test_settings_mirror_the_reference_names_and_errors():
    from pgm_jax_b200.forcefield import MDSettings

    s = MDSettings()
    assert (s.cutoff, s.ewald_beta, s.pme_order, s.dipole_tol, s.max_iter, s.predictor, s.peek) == (0.9, 4.0, 6, 1e-5, 50, "mu4", 0.65)
    assert s.replace(dipole_tol=1e-6).dipole_tol == 1e-6
    with pytest.raises(TypeError):
        s.replace(nonsense=1)
    assert s.replace(iel="0scf").iel == "0scf"  # extended-Lagrangian dipoles are in this engine
    with pytest.raises(ValueError):
        s.replace(long_range="ips")  # a reference setting outside this path
    with pytest.raises(ValueError):
        s.replace(iel="xl")
    with pytest.raises(ValueError):
        MDSettings(elec="qq")


def test_pgm3p25_water_parameters():
    from pgm_jax_b200.systems import pgm3p25_water, water_geometry

    m = pgm3p25_water()
    assert np.allclose(m.q, [-2.04056220, 1.02028110, 1.02028110]) and abs(m.q.sum()) < 1e-12
    assert np.allclose(m.radius, [0.0605150752, 0.0536231183, 0.0536231183])
    assert np.allclose(m.alpha, [1.11765163e-3, 0.329630770e-3, 0.329630770e-3])
    A, B = 5.81935564e5, 5.94825035e2
    rmin_nm, eps_kj = (2 * A / B) ** (1 / 6) * 0.1, B * B / (4 * A) * 4.184
    assert abs(2 * m.lj_rmin_half[0] - rmin_nm) < 1e-12 and abs(m.lj_sqrt_eps[0] ** 2 - eps_kj) < 1e-12
    w = water_geometry()
    assert abs(np.linalg.norm(w[1] - w[0]) - 0.09572) < 1e-12
    assert abs(np.degrees(np.arccos(np.dot(w[1], w[2]) / 0.09572**2)) - 104.52) < 1e-9


def test_rigid_bodies_reconstruct_positions():
    from pgm_jax_b200.md import rigid_bodies
    from pgm_jax_b200.systems import small_box

    s, pos, H = small_box(0)
    com, quat, body, I = rigid_bodies(s, pos, H)
    for m in range(s.nmol):
        w, x, y, z = quat[m]
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        a0, a1 = s.mol_start[m], s.mol_start[m + 1]
        rec = com[m] + body[a0:a1] @ R.T
        d = rec - pos[a0:a1]
        for c in (2, 1, 0):
            d = d - np.round(d[:, c] / H[c, c])[:, None] * H[c]
        assert np.abs(d).max() < 1e-12
        assert np.all(I[m] > 0)


def test_step_bytes_formula():
    import bench

    # 3.76 M pairs, 6 iterations, 96^3: about 1.1 GB per step (the 4096-water example)
    b = bench.bytes_per_step(12288, 3.76e6, 6, 96)
    assert 1.0e9 < b < 1.2e9


def test_local_preconditioner_settings_are_checked():
    """local_niter 0..8, local_cut below the cutoff, not with iel."""
    from pgm_jax_b200.forcefield import MDSettings

    with pytest.raises(ValueError):
        MDSettings(local_niter=1, local_cut=0.95)
    with pytest.raises(ValueError):
        MDSettings(local_niter=1, iel="0scf")
    with pytest.raises(ValueError):
        MDSettings(local_niter=9)
