"""Monte Carlo barostat on the engine: accepted moves scale the box and the molecular centres and
keep orientations and momenta, the new state's energy is the trial energy, rejected moves change
nothing, and NPT steps run."""

import numpy as np
import pytest
import torch
from conftest import SMALL_BOX_SETTINGS

pytestmark = pytest.mark.gpu


def make_md(system, pos, H):
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import RigidMD

    st = dict(SMALL_BOX_SETTINGS, dipole_tol=1e-9, max_iter=200)
    ff = PGMForceField(system, H, MDSettings(precision="double", **st))
    return RigidMD(ff, pos, H, temperature=300.0, dt_fs=0.5, gamma_ps=5.0, seed=3)


def snapshot(md):
    return {k: getattr(md, k).clone() for k in ("pos", "com", "quat", "mom", "angmom", "box")} | {"mu": md.ind.mu.clone()}


def test_accepted_and_rejected_moves(small_box_system):
    from pgm_jax_b200.barostat import MonteCarloBarostat

    s, pos, H = small_box_system
    md = make_md(s, pos, H)
    for _ in range(3):
        md.step()
    baro = MonteCarloBarostat(md, pressure=1.0, every=5, seed=1)
    V = baro.volumes()[0]
    # rejected (log u = +inf): nothing of the MD state changes
    before = snapshot(md)
    acc = baro.attempt(dV=[0.02 * V], log_u=[np.inf])
    assert not acc[0]
    after = snapshot(md)
    for k in before:
        assert torch.equal(before[k], after[k]), k
    # accepted (log u = -inf): box and centres scaled by s, orientations and momenta kept
    dV = -0.02 * V
    s3 = np.cbrt((V + dV) / V)
    count0 = int(md.ind.count[0])
    acc = baro.attempt(dV=[dV], log_u=[-np.inf])
    assert acc[0]
    after = snapshot(md)
    assert torch.allclose(after["box"], before["box"] * s3, rtol=0, atol=1e-14)
    assert torch.allclose(after["com"], before["com"] * s3, rtol=0, atol=1e-12)
    for k in ("quat", "mom", "angmom"):
        assert torch.equal(before[k], after[k]), k
    shift = after["pos"] - before["pos"]
    mols = torch.tensor(np.repeat(np.arange(md.nmol), np.diff(md._keep[0])), device=md.dev)
    assert torch.allclose(shift, (s3 - 1.0) * before["com"][mols], rtol=0, atol=1e-12)
    assert abs(baro.volumes()[0] - (V + dV)) <= 1e-9 * V
    # the forces were recomputed at the new state: its energy is the trial energy (same dipoles)
    e_after = float(md.result.energy["total"][0])
    e_trial, _, _, _ = md.ff.energy(md.pos, md.box, None, md.ind)
    assert abs(e_after - float(e_trial[0])) <= 1e-8 * abs(e_after)
    assert int(md.ind.count[0]) == count0 + 1 and int(md.ff._status[0]) == 0


def test_npt_steps_run(small_box_system):
    """30 captured steps with a move every 5: finite energies, clean status, a changed volume."""
    from pgm_jax_b200.barostat import MonteCarloBarostat

    s, pos, H = small_box_system
    md = make_md(s, pos, H)
    md.step()
    md.capture()
    baro = MonteCarloBarostat(md, pressure=1.0, every=5, seed=2)
    V0 = baro.volumes()[0]
    baro.run(30)
    md.stream.synchronize()
    assert int(baro.total_tries[0]) == 6
    assert np.isfinite(float(md.result.energy["total"][0])) and int(md.ff._status[0]) == 0
    if baro.total_accepted[0] > 0:
        assert baro.volumes()[0] != V0
    e = md.energy()
    assert np.isfinite(e["total"][0])
