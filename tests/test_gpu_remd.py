"""Replica exchange on the GPU: uneven boxes and temperature replicas in one batched engine, the
captured MD step reading the exchanged temperatures, momenta rescaled by sqrt(T_new / T_old)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_replicas_beside_uneven_boxes_in_one_launch():
    from pgm_jax_b200.forcefield import MDSettings, PGMForceField
    from pgm_jax_b200.md import KB, RigidMD
    from pgm_jax_b200.remd import ReplicaExchange, RigidReplicas, geometric_ladder
    from pgm_jax_b200.systems import water_box

    boxes = [water_box(4, 1.25, seed=11), water_box(5, 1.55, seed=12)] + [water_box(4, 1.25, seed=20 + k) for k in range(4)]
    grids = [(32, 32, 32), (36, 36, 36)] + [(32, 32, 32)] * 4
    st = MDSettings(precision="mixed", cutoff=0.6, ewald_beta=5.0, dipole_tol=1e-6, max_iter=100)
    ff = PGMForceField([b[0] for b in boxes], [b[2] for b in boxes], st, pme_grids=grids)
    T = geometric_ladder(280.0, 400.0, 4)
    md = RigidMD(ff, np.concatenate([b[1] for b in boxes]), np.stack([b[2] for b in boxes]),
                 temperature=[300.0, 300.0] + list(T), dt_fs=1.0, gamma_ps=5.0, seed=3)
    rex = ReplicaExchange(RigidReplicas(md, systems=[2, 3, 4, 5]), T, seed=1)
    for _ in range(3):
        md.step()
    md.capture()
    n_round = 12
    for _ in range(n_round):
        md.run(20)
        ke0, t0 = md.kinetic(), md.temps.copy()
        rex.exchange()
        ke1, t1 = md.kinetic(), md.temps.copy()
        assert np.allclose(t1[2:], rex.temperature_of_system()) and np.allclose(t1[:2], 300.0)
        assert np.allclose(md.kT.cpu().numpy(), KB * t1, rtol=1e-15)
        assert np.allclose(ke1 / ke0, t1 / t0, rtol=1e-12)  # swapped systems rescaled, the others untouched
        assert not np.any(md.result.status.cpu().numpy() & 0x6)
    assert rex.stats.attempts.sum() == 2 * sum(len(range(k & 1, 3, 2)) for k in range(n_round))
    # the batch evaluates every system as it would alone
    md.stream.synchronize()
    rb = ff.compute(md.pos, md.box)
    for k in (1, 3):
        sl = slice(int(ff.offsets[k]), int(ff.offsets[k + 1]))
        f1 = PGMForceField(boxes[k][0], boxes[k][2], st, pme_grids=[grids[k]])
        r1 = f1.compute(md.pos[sl], md.box[k])
        e1, eb = float(r1.energy["total"][0]), float(rb.energy["total"][k])
        assert abs(eb - e1) <= 1e-6 * abs(e1), (k, eb, e1)
        assert float((rb.forces[sl] - r1.forces).norm() / r1.forces.norm()) <= 1e-5
