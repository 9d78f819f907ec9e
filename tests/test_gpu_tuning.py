"""The autotuner's kernel variants (GPU): every choice of lanes per row in the CG matvec's row
stream, of blocks per SM in the force pass, of the order of the CG sweep's concurrent parts (the
row field of p, or of z combined with the previous direction's) and of the row field's grid beside
the FFT chain (all SMs, or 1 or 2 blocks per SM at the highest priority) computes the same step (FP64: only
the order of additions changes), and the first direct step of a handle times them and keeps the
fastest."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = [(32, 3, 0, 0), (16, 2, 1, 1), (8, 4, 0, 2), (16, 3, 1, 2), (8, 2, 1, 0), (32, 4, 1, 1), (32, 3, 0, 1)]


def _box():
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(8, 2.483, seed=3)
    st = dict(cutoff=0.9, ewald_beta=4.0, pme_grid=(48, 48, 48), pme_order=6, dipole_tol=1e-8, max_iter=100)
    return s, pos, H, st


@pytest.mark.parametrize("prec", ["double", "mixed"])
def test_every_variant_computes_the_same_step(prec):
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField

    s, pos, H, st = _box()
    out = []
    for lanes, blocks, early, grid in VARIANTS:
        ff = PGMForceField(s, H, MDSettings(precision=prec, **st))
        ff.set_tuning(lanes, blocks, early, grid)
        r = ff.compute(pos, H)
        t = ff.tuning()
        assert (t["rowfield_lanes"], t["forces_blocks_per_sm"], t["sweep_early"], t["rowfield_grid"]) == (
            lanes, blocks, early, grid) and not t["tuned"]
        out.append((float(r.energy["total"][0]), r.forces.cpu().numpy(), r.induction.mu.cpu().numpy(), int(r.iterations[0])))
    e0, f0, m0, i0 = out[0]
    tol = 1e-12 if prec == "double" else 1e-6
    for (e, f, m, it), v in zip(out[1:], VARIANTS[1:]):
        assert abs(e - e0) <= tol * abs(e0), (v, e, e0)
        assert np.abs(f - f0).max() <= (1e-10 if prec == "double" else 1e-4) * np.abs(f0).max(), v
        assert np.abs(m - m0).max() <= (1e-10 if prec == "double" else 1e-4) * np.abs(m0).max(), v
        assert abs(it - i0) <= (0 if prec == "double" else 1), (v, it, i0)


def test_first_direct_step_autotunes():
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField

    s, pos, H, st = _box()
    ff = PGMForceField(s, H, MDSettings(precision="mixed", **st))
    assert not ff.tuning()["tuned"]
    ff.compute(pos, H)
    t = ff.tuning()
    assert t["tuned"] and t["rowfield_lanes"] in (32, 16, 8) and t["forces_blocks_per_sm"] in (2, 3, 4)
    assert all(ms > 0 for ms in t["rowfield_ms"] + t["forces_ms"] + t["sweep_ms"])
    assert t["sweep_early"] == (1 if t["sweep_ms"][1] < t["sweep_ms"][0] else 0)
    assert all(ms > 0 for ms in t["grid_ms"]) and t["grid_ms"][t["rowfield_grid"]] == min(t["grid_ms"])
    assert t["rowfield_ms"][[32, 16, 8].index(t["rowfield_lanes"])] == min(t["rowfield_ms"])
    # a second handle of the same shape takes the choice from the cache
    ff2 = PGMForceField(s, H, MDSettings(precision="mixed", **st))
    ff2.compute(pos, H)
    t2 = ff2.tuning()
    assert t2["tuned"] and t2["from_cache"] and t2["rowfield_lanes"] == t["rowfield_lanes"]
