"""Path-integral MD on the GPU: the normal-mode free step against the NumPy restatement, the
q-TIP4P/F forces against finite differences, RPMD conserving the ring-polymer Hamiltonian, graph
replays equal to direct steps, and the PILE thermostat holding every internal mode at T."""

import ctypes as C
import math

import numpy as np
import pytest
import torch

import pimd_oracle as PO

pytestmark = pytest.mark.gpu


def _t(a, dt=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_free_step_matches_numpy():
    from pgm_jax_b200 import _lib
    from pgm_jax_b200.pimd import RingPolymer

    lib = _lib.load()
    for P in (1, 6, 8, 32):
        ring = RingPolymer(P, 300.0)
        rng = np.random.default_rng(P)
        n = 37
        q, p = rng.normal(scale=0.01, size=(P, n, 3)), rng.normal(size=(P, n, 3))
        m = rng.uniform(1, 16, size=n)
        dq, dp = _t(q.reshape(-1, 3)), _t(p.reshape(-1, 3))
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        keep = [_t(ring.C), _t(ring.omega), _t(np.zeros(P)), _t(m)]  # alive until the kernel has run
        _lib.check(lib.pgm_pimd_free_thermostat(None, P, n, *[_p(k) for k in keep], 0.0005, ring.kT_P, 1, _p(cnt), _p(dq), _p(dp)))
        torch.cuda.synchronize()
        qr, pr = PO.free_step(q, p, ring.C, ring.omega, m, 0.0005)
        assert np.abs(dq.cpu().numpy().reshape(P, n, 3) - qr).max() <= 1e-13
        assert np.abs(dp.cpu().numpy().reshape(P, n, 3) - pr).max() <= 1e-11 * np.abs(pr).max()
        assert int(cnt.item()) == 1


def test_pile_g_centroid_factor_and_scaled_free_step():
    """PILE-G on the device: the centroid kinetic energy and Bussi factor equal the restatement for
    the draws the kernel reports, and the free step with the centroid rescaled equals the NumPy one."""
    from pgm_jax_b200 import _lib
    from pgm_jax_b200.pimd import RingPolymer

    lib = _lib.load()
    P, n, dt, tau = 8, 37, 0.0005, 0.2
    ring = RingPolymer(P, 300.0)
    rng = np.random.default_rng(11)
    q, p = rng.normal(scale=0.01, size=(P, n, 3)), rng.normal(size=(P, n, 3))
    m = rng.uniform(1, 16, size=n)
    dq, dp = _t(q.reshape(-1, 3)), _t(p.reshape(-1, 3))
    cnt = torch.full((1,), 7, dtype=torch.int64, device="cuda")
    work = torch.zeros(4, dtype=torch.float64, device="cuda")
    keep = [_t(ring.C), _t(ring.omega), _t(np.zeros(P)), _t(m)]
    _lib.check(lib.pgm_pimd_centroid_bussi(None, P, n, _p(keep[0]), _p(keep[3]), dt, ring.kT_P, tau, 5, _p(cnt), _p(dp), _p(work)))
    torch.cuda.synchronize()
    K, alpha, r1, S = work.cpu().numpy()
    assert abs(K - PO.centroid_kinetic(p, ring.C, m)) <= 1e-12 * K
    assert S > 0 and abs(alpha - PO.bussi_factor(K, ring.kT_P, 3 * n, dt, tau, r1, S)) <= 1e-13
    _lib.check(lib.pgm_pimd_free_thermostat_scaled(None, P, n, *[_p(k) for k in keep], dt, ring.kT_P, 5, _p(cnt), _p(dq), _p(dp),
                                                   C.c_void_p(work.data_ptr() + 8)))
    torch.cuda.synchronize()
    qr, pr = PO.free_step_centroid_scaled(q, p, ring.C, ring.omega, m, dt, alpha)
    assert np.abs(dq.cpu().numpy().reshape(P, n, 3) - qr).max() <= 1e-13
    assert np.abs(dp.cpu().numpy().reshape(P, n, 3) - pr).max() <= 1e-11 * np.abs(pr).max()
    assert int(cnt.item()) == 8
    # the device draws: R1 ~ N(0, 1) and S ~ chi^2(3n - 1) over many steps
    r1s, ss = [], []
    for step in range(400):
        cnt.fill_(1000 + step)
        _lib.check(lib.pgm_pimd_centroid_bussi(None, P, n, _p(keep[0]), _p(keep[3]), dt, ring.kT_P, tau, 5, _p(cnt), _p(dp),
                                               _p(work)))
        w = work.cpu().numpy()
        r1s.append(w[2]); ss.append(w[3])
    r1s, ss = np.array(r1s), np.array(ss)
    dof1 = 3 * n - 1
    assert abs(r1s.mean()) < 4 / np.sqrt(len(r1s)) and abs(r1s.std() - 1) < 0.15
    assert abs(ss.mean() - dof1) < 4 * np.sqrt(2 * dof1 / len(ss)) and abs(ss.var() / (2 * dof1) - 1) < 0.3


def test_water_bonded_forces():
    from pgm_jax_b200 import _lib
    from pgm_jax_b200.pimd import QTIP4PF

    lib = _lib.load()
    rng = np.random.default_rng(3)
    nw = 20
    base = np.array([[0.0, 0.0, 0.0], [0.0957, 0.0, 0.0], [-0.024, 0.0927, 0.0]])
    R = np.concatenate([base + rng.normal(scale=0.006, size=(3, 3)) + 0.5 * k for k in range(nw)])
    prm = np.array([QTIP4PF["D"], QTIP4PF["alpha"], QTIP4PF["r_eq"], QTIP4PF["k_theta"], math.radians(QTIP4PF["theta_eq"])])
    f = torch.zeros((3 * nw, 3), dtype=torch.float64, device="cuda")
    e = torch.zeros(2, dtype=torch.float64, device="cuda")
    first = _t(np.arange(nw) * 3, torch.int32)
    msys = _t(np.arange(nw) % 2, torch.int32)
    dR = _t(R)
    _lib.check(lib.pgm_water_bonded(None, nw, _p(first), _p(msys), _p(dR), C.c_void_p(prm.ctypes.data), _p(f), _p(e)))
    torch.cuda.synchronize()
    F = f.cpu().numpy()
    E = np.zeros(2)
    for k in range(nw):
        ek, fk = PO.qtip4pf_forces(R[3 * k:3 * k + 3], prm)
        E[k % 2] += ek
        assert np.abs(F[3 * k:3 * k + 3] - fk).max() <= 1e-5 * max(1.0, np.abs(fk).max())
    assert np.allclose(e.cpu().numpy(), E, rtol=1e-12)


def _pimd(mode, P, prec, seed=1, dt_fs=0.25, n_side=3, edge=0.95, centroid="l"):
    from pgm_jax_b200.forcefield import MDSettings
    from pgm_jax_b200.pimd import PIMD
    from pgm_jax_b200.systems import water_box

    s, pos, H = water_box(n_side, edge, seed=seed)
    st = MDSettings(precision=prec, cutoff=0.45, ewald_beta=7.0, pme_grid=(32, 32, 32), dipole_tol=1e-10 if prec == "double" else 1e-6,
                    max_iter=200)
    return PIMD(s, pos, H, st, beads=P, temperature=300.0, dt_fs=dt_fs, mode=mode, seed=seed, centroid=centroid)


def test_rpmd_conserves_the_ring_polymer_hamiltonian_and_graphs_replay_steps():
    pm = _pimd("rpmd", 4, "double")
    H0 = pm.estimators()
    hs, kes = [], []
    for _ in range(60):
        pm.step()
        e = pm.estimators()
        hs.append(e["hamiltonian"])
        kes.append(e["ke_beads"])
    assert np.std(hs) < 0.02 * np.std(kes), (np.std(hs), np.std(kes))
    assert abs(hs[-1] - H0["hamiltonian"]) < 0.05 * np.std(kes) + 1e-3 * abs(H0["hamiltonian"])
    # graph replays continue the same trajectory as direct steps
    q0, p0 = pm.q.clone(), pm.p.clone()
    ind0 = [t.clone() for t in (pm.ind.mu, pm.ind.hist, pm.ind.count, pm.ind.norm)]
    f0 = pm.forces.clone()
    for _ in range(4):
        pm.step()
    pm.stream.synchronize()
    qd = pm.q.clone()
    pm.q.copy_(q0); pm.p.copy_(p0); pm.forces.copy_(f0)
    for dst, src in zip((pm.ind.mu, pm.ind.hist, pm.ind.count, pm.ind.norm), ind0):
        dst.copy_(src)
    torch.cuda.synchronize()
    pm.capture()
    pm.q.copy_(q0); pm.p.copy_(p0); pm.forces.copy_(f0)
    for dst, src in zip((pm.ind.mu, pm.ind.hist, pm.ind.count, pm.ind.norm), ind0):
        dst.copy_(src)
    torch.cuda.synchronize()
    pm.run(4)
    pm.stream.synchronize()
    assert float((pm.q - qd).abs().max()) <= 1e-9


def test_pile_holds_internal_modes_at_temperature():
    pm = _pimd("pimd", 8, "mixed", dt_fs=0.5, n_side=4, edge=1.25)
    pm.capture()
    pm.run(100)
    t = []
    for _ in range(60):
        pm.run(5)
        t.append(pm.estimators()["t_modes"])
    t = np.array(t)
    internal = t[:, 1:].mean()
    assert abs(internal / 300.0 - 1.0) < 0.05, t.mean(0)
    assert not int(pm.result.status.max()) & 0x6


def test_pile_g_holds_every_mode_at_temperature():
    """PILE-G: Bussi's centroid rescaling (tight, tau 0.01 ps, against the heat the relaxing lattice
    start releases) and the internal modes' Langevin keep the centroid and the internal modes near T
    once the start has relaxed (0.4 ps)."""
    pm = _pimd("pimd", 8, "mixed", dt_fs=0.5, n_side=4, edge=1.25, centroid="g")
    pm.tau0 = 0.01
    pm.capture()
    pm.run(800)
    t = []
    for _ in range(60):
        pm.run(5)
        t.append(pm.estimators()["t_modes"])
    t = np.array(t)
    assert abs(t[:, 1:].mean() / 300.0 - 1.0) < 0.05, t.mean(0)
    assert abs(t[:, 0].mean() / 300.0 - 1.0) < 0.1, t[:, 0].mean()
    assert float(pm.bussi_work[1]) > 0 and not int(pm.result.status.max()) & 0x6
