"""The FP64 CPU oracle against the reference's golden vectors and physics checks (no GPU)."""

import numpy as np
import pytest
from conftest import SMALL_BOX_SETTINGS

import oracle as O


@pytest.fixture(scope="module")
def small(small_box_system, golden_small_box):
    s, pos, H = small_box_system
    assert np.array_equal(pos, golden_small_box["pos"]) and np.array_equal(H, golden_small_box["box"])
    o = O.Oracle(s, SMALL_BOX_SETTINGS)
    return s, pos, H, o, o.compute(pos, H)


def test_oracle_matches_reference_golden_double(small, golden_small_box):
    """Energies, forces, dipoles, CG iterations and residual of ff_small_box (float64)."""
    g = golden_small_box
    _, _, _, _, r = small
    for k in ("elec", "vdw", "total"):
        ref = float(g[f"double.energy.{k}"])
        assert abs(r["energy"][k] - ref) <= 1e-10 * abs(ref), (k, r["energy"][k], ref)
    assert r["iterations"] == int(g["double.iterations"])
    assert abs(r["residual"] - float(g["double.residual"])) <= 1e-6 * float(g["double.residual"])
    F = g["double.forces"]
    assert np.abs(r["forces"] - F).max() <= 1e-8 * np.abs(F).max()
    mu = g["double.mu"]
    assert np.abs(r["mu"] - mu).max() <= 1e-9 * np.abs(mu).max()


def test_oracle_strain_matches_reference_golden(small, golden_small_box):
    """The analytic molecular virial equals the reference's autodiff strain derivative."""
    W = golden_small_box["double.strain"]
    assert np.abs(small[4]["virial"] - W).max() <= 1e-7 * np.abs(W).max()


def test_erf_kernels_series_and_closed_form_agree_at_switch():
    a = 9.0
    for r in (0.99 / a, 1.01 / a, 0.05, 0.3):
        B = O.erf_kernels(a, r)
        from math import erf, exp, pi, sqrt

        assert abs(B[0] - erf(a * r) / r) < 1e-12 * B[0]
        B1 = (erf(a * r) / r - 2 * a / sqrt(pi) * exp(-a * a * r * r)) / (r * r)
        assert abs(B[1] - B1) < 1e-9 * abs(B1)
    lo, hi = O.erf_kernels(a, (1 - 1e-9) / a), O.erf_kernels(a, (1 + 1e-9) / a)
    assert np.allclose(lo, hi, rtol=1e-7)


@pytest.mark.parametrize("order", [4, 6, 8])
def test_bspline_partition_of_unity_and_derivatives(order):
    for f in (0.0, 0.3, 0.77):
        t, d, s = O.bspline(f, order)
        assert abs(t.sum() - 1) < 1e-14 and abs(d.sum()) < 1e-13 and abs(s.sum()) < 1e-12
        h = 1e-6
        tp, dp, _ = O.bspline(f + h, order)
        tm, dm, _ = O.bspline(f - h, order) if f > 0 else O.bspline(f, order)
        den = 2 * h if f > 0 else h
        assert np.allclose((tp - tm) / den, d, atol=1e-6)
        assert np.allclose((dp - dm) / den, s, atol=1e-5)


def test_oracle_forces_equal_central_differences(small):
    """Forces at fixed mu against central differences of the energy (test_md.py:51 analogue)."""
    s, pos, H, o, r = small
    h = 1e-6
    for a, k in [(0, 0), (5, 1), (40, 2), (77, 0)]:
        d = np.zeros_like(pos)
        d[a, k] = h
        fd = -(o.energy_fixed_mu(pos + d, H, r["mu"])["total"] - o.energy_fixed_mu(pos - d, H, r["mu"])["total"]) / (2 * h)
        assert abs(fd - r["forces"][a, k]) < 1e-5 * max(1.0, abs(fd)), (a, k, fd, r["forces"][a, k])


def test_oracle_strain_trace_equals_isotropic_scaling(small):
    """Trace of the virial against scaling box and molecular centres (test_md.py:119 analogue)."""
    s, pos, H, o, r = small
    m = s.masses
    com = np.array([np.average(pos[s.mol == k], 0, weights=m[s.mol == k]) for k in range(s.nmol)])
    h = 1e-6

    def e(x):
        return o.energy_fixed_mu(pos + (x * com)[s.mol], H * (1 + x), r["mu"])["total"]

    fd = (e(h) - e(-h)) / (2 * h)
    vol = abs(np.linalg.det(H))
    M = [np.sum(s.lj_sqrt_eps * s.lj_rmin_half**k) for k in range(7)]
    from math import comb, pi

    tail = -2 * pi * 2 * sum(comb(6, k) * M[k] * M[6 - k] for k in range(7)) / (3 * vol * 0.6**3)
    assert abs(fd - 3 * tail - np.trace(r["virial"])) < 1e-5 * max(1.0, abs(fd))


@pytest.mark.parametrize("elec", ["q", "qp", "qi"])
def test_oracle_elec_levels(small_box_system, elec):
    """q / qp / qi run, give no CG without induction, and differ from qpi."""
    s, pos, H = small_box_system
    o = O.Oracle(s, dict(SMALL_BOX_SETTINGS, elec=elec))
    r = o.compute(pos, H)
    if "i" not in elec:
        assert r["iterations"] == 0 and np.all(r["mu"] == 0)
    else:
        assert r["iterations"] > 0
    assert np.isfinite(r["energy"]["total"])


def test_oracle_forces_without_permanent_dipoles_are_pure_charge(small_box_system):
    """At level "q" the covalent frames carry no dipole, so the forces are central differences of E."""
    s, pos, H = small_box_system
    o = O.Oracle(s, dict(SMALL_BOX_SETTINGS, elec="q"))
    r = o.compute(pos, H)
    h = 1e-6
    for a, k in [(0, 0), (7, 2)]:
        d = np.zeros_like(pos)
        d[a, k] = h
        fd = -(o.energy_fixed_mu(pos + d, H, r["mu"])["total"] - o.energy_fixed_mu(pos - d, H, r["mu"])["total"]) / (2 * h)
        assert abs(fd - r["forces"][a, k]) < 1e-5 * max(1.0, abs(fd))


def test_oracle_split_rows(small):
    """Split rows (elec_cutoff < cutoff, forcefield.py:44-58): elec_cutoff = cutoff changes nothing;
    below it the LJ term keeps every pair inside the cutoff and the forces stay the central
    differences of the energy."""
    s, pos, H, o, r = small
    same = O.Oracle(s, dict(SMALL_BOX_SETTINGS, elec_cutoff=SMALL_BOX_SETTINGS["cutoff"])).compute(pos, H)
    assert same["energy"]["total"] == r["energy"]["total"] and np.array_equal(same["forces"], r["forces"])
    os_ = O.Oracle(s, dict(SMALL_BOX_SETTINGS, elec_cutoff=0.45))
    rs = os_.compute(pos, H)
    assert abs(rs["energy"]["vdw"] - r["energy"]["vdw"]) <= 1e-12 * abs(r["energy"]["vdw"])
    assert abs(rs["energy"]["elec"] - r["energy"]["elec"]) > 1e-6 * abs(r["energy"]["elec"])
    h = 1e-6
    for a, k in [(0, 0), (40, 2)]:
        d = np.zeros_like(pos)
        d[a, k] = h
        fd = -(os_.energy_fixed_mu(pos + d, H, rs["mu"])["total"] - os_.energy_fixed_mu(pos - d, H, rs["mu"])["total"]) / (2 * h)
        assert abs(fd - rs["forces"][a, k]) < 1e-5 * max(1.0, abs(fd)), (a, k, fd, rs["forces"][a, k])


def test_oracle_matches_reference_golden_pgm3p25_512(pgm3p25_512_system, golden_pgm3p25_512):
    """512 pGM3P-25 waters of the reference's examples/water512 frame at the default settings
    (regression case ff_pgm3p25_512): the parameters, the truncated-octahedron box and the 30^3
    mesh of every pGM3P-25 workload, pinned to the reference's float64 output."""
    from conftest import PGM3P25_512_SETTINGS

    from pgm_jax_b200.systems import grid_size

    g = golden_pgm3p25_512
    assert grid_size(g["box"], 0.08) == PGM3P25_512_SETTINGS["pme_grid"]
    r = O.Oracle(pgm3p25_512_system, PGM3P25_512_SETTINGS).compute(g["pos"], g["box"])
    for k in ("elec", "vdw", "total"):
        ref = float(g[f"double.energy.{k}"])
        assert abs(r["energy"][k] - ref) <= 1e-10 * abs(ref), (k, r["energy"][k], ref)
    assert r["iterations"] == int(g["double.iterations"])
    F, mu = g["double.forces"], g["double.mu"]
    assert np.sqrt(np.sum((r["forces"] - F) ** 2) / np.sum(F**2)) <= 1e-8
    assert np.sqrt(np.sum((r["mu"] - mu) ** 2) / np.sum(mu**2)) <= 1e-8
    W = g["double.strain"]
    assert np.abs(r["virial"] - W).max() <= 1e-6 * np.abs(W).max()


def test_oracle_local_preconditioner_same_solution_fewer_iterations(pgm3p25_512_system, golden_pgm3p25_512):
    """The local preconditioner (inner CG on the row entries closer than local_cut, flexible PCG;
    forcefield.py:1766-1811) converges to the same dipoles as Jacobi PCG in fewer outer
    iterations, and local_niter = 0 is Jacobi itself (the golden's 9 iterations)."""
    from conftest import PGM3P25_512_SETTINGS

    g = golden_pgm3p25_512
    out = {}
    for ni in (0, 2):
        st = dict(PGM3P25_512_SETTINGS, dipole_tol=1e-9, max_iter=100, local_cut=0.3, local_niter=ni)
        out[ni] = O.Oracle(pgm3p25_512_system, st).compute(g["pos"], g["box"])
    assert out[2]["iterations"] < out[0]["iterations"]
    assert np.abs(out[2]["mu"] - out[0]["mu"]).max() <= 1e-7 * np.abs(out[0]["mu"]).max()
    assert abs(out[2]["energy"]["total"] - out[0]["energy"]["total"]) <= 1e-10 * abs(out[0]["energy"]["total"])
    st = dict(PGM3P25_512_SETTINGS, local_niter=0)
    assert O.Oracle(pgm3p25_512_system, st).compute(g["pos"], g["box"])["iterations"] == int(g["double.iterations"])


def test_oracle_matches_pmemd_pgm(pgm3p25_512_system, golden_pgm3p25_512, golden_pmemd_pbc_512):
    """The independent pmemd-pgm (Amber) single point that pGM-JAX keeps for validation
    (data/validation/amber_ref/pmemd_pbc): PME 72^3 order 8, 10 A cutoff, ewald 0.38 / A, no LJ tail,
    on the water512 frame.  EELEC (Tinker's Coulomb constant) to 1e-9 relative (mdout prints 4
    decimals of 5e5), VDWAALS to its printed digits, forces to the FP32 precision pmemd stores them
    in, induced dipoles to 1e-10 e A RMS."""
    from conftest import PMEMD_PBC_SETTINGS, pmemd_compare

    g = golden_pgm3p25_512
    r = O.Oracle(pgm3p25_512_system, PMEMD_PBC_SETTINGS).compute(g["pos"], g["box"])
    re_ = O.Oracle(pgm3p25_512_system, dict(PMEMD_PBC_SETTINGS, vdw="none")).compute(g["pos"], g["box"])
    de, dv, df, dmu = pmemd_compare(r["energy"]["elec"], r["energy"]["vdw"], re_["forces"], r["forces"], r["mu"],
                                    golden_pmemd_pbc_512)
    assert de <= 1e-9, de
    assert dv <= 1e-4, dv
    assert df <= 2e-6, df
    assert dmu <= 1e-10, dmu

