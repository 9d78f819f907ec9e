"""ctypes front end of the FP64 CPU oracle -- TEST INFRASTRUCTURE, NOT THE PRODUCT.

The oracle (pgm_oracle.c) restates pGM-JAX's PGMForceField.compute (pgm_jax/md/forcefield.py:2489)
in plain FP64 C.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as
the checker; the product path never calls it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libpgm_oracle.so")

_i = C.c_int
_d = C.c_double
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int)


class _Sys(C.Structure):
    _fields_ = [
        ("n", _i), ("nmol", _i), ("mol_start", _pi), ("q", _pd), ("radius", _pd), ("alpha", _pd),
        ("rmin_half", _pd), ("sqrt_eps", _pd), ("mass", _pd), ("ncov", _i), ("cov_i", _pi), ("cov_j", _pi),
        ("cov_c", _pd),
    ]


class _Set(C.Structure):
    _fields_ = [
        ("perm", _i), ("induce", _i), ("lj", _i), ("lj_lrc", _i), ("cutoff", _d), ("beta", _d), ("K", _i * 3),
        ("order", _i), ("tol", _d), ("max_iter", _i), ("predictor", _i), ("fused", _i), ("norm_refresh", _i),
        ("peek", _d), ("nthreads", _i), ("elec_cutoff", _d),
        ("iel", _i), ("iel_order", _i), ("iel_kappa", _d), ("iel_alpha", _d), ("iel_omega", _d), ("iel_precond", _i),
        ("iel_iter", _i), ("iel_shadow", _i), ("local_cut", _d), ("local_niter", _i),
    ]


class _Res(C.Structure):
    _fields_ = [
        ("elec", _d), ("vdw", _d), ("total", _d), ("virial", _d * 9), ("iterations", _i), ("residual", _d),
        ("pairs", C.c_longlong),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP) if needed; return the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        for name in ("pgmo_compute", "pgmo_energy_fixed_mu", "pgmo_field", "pgmo_perm_dipoles", "pgmo_compute_iel",
                     "pgmo_iel_len"):
            getattr(_lib, name).restype = _i
        _lib.pgmo_erf_kernels.restype = None
        _lib.pgmo_bspline.restype = None
    return _lib


def _p(a, t=_pd):
    return a.ctypes.data_as(t)


class Oracle:
    """FP64 oracle of one system with fixed settings (numpy in, numpy out).

    settings: a dict with the flat names of MDSettings (elec, vdw, lj_lrc, cutoff, ewald_beta,
    pme_grid, pme_order, dipole_tol, max_iter, predictor, fused, norm_refresh, peek).
    """

    def __init__(self, system, settings: dict, nthreads: int = 0) -> None:
        self.sys = system
        self._keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(x, dtype=dt)
            self._keep.append(a)
            return a

        s = system
        self._s = _Sys(
            s.n, s.nmol, _p(arr(s.mol_start, np.int32), _pi), _p(arr(s.q, float)), _p(arr(s.radius, float)),
            _p(arr(s.alpha, float)), _p(arr(s.lj_rmin_half, float)), _p(arr(s.lj_sqrt_eps, float)),
            _p(arr(s.masses, float)), len(s.cov_i), _p(arr(s.cov_i, np.int32), _pi), _p(arr(s.cov_j, np.int32), _pi),
            _p(arr(s.cov_c, float)),
        )
        st = dict(settings)
        elec = st.get("elec", "qpi")
        pred = {"none": 0, "mu1": 1, "mu3": 3, "mu4": 4}[st.get("predictor", "mu4")]
        K = st["pme_grid"]
        self._set = _Set(
            int("p" in elec), int("i" in elec), int(st.get("vdw", "lj") == "lj"), int(st.get("lj_lrc", True)),
            float(st.get("cutoff", 0.9)), float(st.get("ewald_beta", 4.0)), (_i * 3)(*K), int(st.get("pme_order", 6)),
            float(st.get("dipole_tol", 1e-5)), int(st.get("max_iter", 50)), pred, int(st.get("fused", True)),
            int(st.get("norm_refresh", 1000)), float(st.get("peek", 0.65)), int(nthreads),
            float(st.get("elec_cutoff") or 0.0),
            {"none": 0, "0scf": 1, "scf": 2}[st.get("iel", "none")], int(st.get("iel_order", 7)),
            float("nan") if st.get("iel_kappa") is None else float(st["iel_kappa"]),
            float("nan") if st.get("iel_alpha") is None else float(st["iel_alpha"]), float(st.get("iel_omega", 1.0)),
            {"jacobi": 0, "block": 1}[st.get("iel_precond", "block")], int(st.get("iel_iter", 1)),
            int(st.get("iel_shadow", True)), float(st.get("local_cut", 0.3)), int(st.get("local_niter", 0)),
        )
        self.iel = st.get("iel", "none") != "none"

    def init_induction(self) -> dict:
        n = self.sys.n
        ind = {"mu": np.zeros((n, 3)), "hist": np.zeros((4, n, 3)), "count": 0, "norm": 1.0}
        if self.iel:
            ind["xl"] = np.zeros((lib().pgmo_iel_len(self._set.iel_order), n, 3))
        return ind

    def compute(self, pos, H, ind: dict | None = None) -> dict:
        """One step: returns energy dict, forces, mu, iterations, residual, virial, and the new state."""
        ind = self.init_induction() if ind is None else {k: (np.array(v) if k in ("mu", "hist", "xl") else v)
                                                          for k, v in ind.items()}
        pos = np.ascontiguousarray(pos, float)
        H = np.ascontiguousarray(H, float)
        mu = np.ascontiguousarray(ind["mu"], float)
        hist = np.ascontiguousarray(ind["hist"], float)
        cnt = C.c_int(int(ind["count"]))
        nrm = C.c_double(float(ind["norm"]))
        F = np.zeros((self.sys.n, 3))
        r = _Res()
        if self.iel:
            xl = np.ascontiguousarray(ind["xl"], float)
            rc = lib().pgmo_compute_iel(C.byref(self._s), C.byref(self._set), _p(pos), _p(H), _p(mu), _p(hist),
                                        C.byref(cnt), C.byref(nrm), _p(xl), _p(F), C.byref(r))
        else:
            rc = lib().pgmo_compute(C.byref(self._s), C.byref(self._set), _p(pos), _p(H), _p(mu), _p(hist), C.byref(cnt),
                                    C.byref(nrm), _p(F), C.byref(r))
        if rc != 0:
            raise RuntimeError(f"oracle compute failed ({rc})")
        return {
            "energy": {"elec": r.elec, "vdw": r.vdw, "total": r.total},
            "forces": F,
            "mu": mu,
            "iterations": r.iterations,
            "residual": r.residual,
            "virial": np.array(r.virial[:]).reshape(3, 3),
            "pairs": r.pairs,
            "induction": dict({"mu": mu, "hist": hist, "count": cnt.value, "norm": nrm.value},
                              **({"xl": xl} if self.iel else {})),
        }

    def energy_fixed_mu(self, pos, H, mu) -> dict:
        out = np.zeros(3)
        lib().pgmo_energy_fixed_mu(C.byref(self._s), C.byref(self._set), _p(np.ascontiguousarray(pos, float)),
                                   _p(np.ascontiguousarray(H, float)), _p(np.ascontiguousarray(mu, float)), _p(out))
        return {"elec": out[0], "vdw": out[1], "total": out[2]}

    def field(self, pos, H, q, d) -> np.ndarray:
        out = np.zeros((self.sys.n, 3))
        qq = None if q is None else np.ascontiguousarray(q, float)
        lib().pgmo_field(C.byref(self._s), C.byref(self._set), _p(np.ascontiguousarray(pos, float)),
                         _p(np.ascontiguousarray(H, float)), _p(qq) if qq is not None else None,
                         _p(np.ascontiguousarray(d, float)), _p(out))
        return out

    def perm_dipoles(self, pos, H) -> np.ndarray:
        out = np.zeros((self.sys.n, 3))
        lib().pgmo_perm_dipoles(C.byref(self._s), _p(np.ascontiguousarray(pos, float)),
                                _p(np.ascontiguousarray(H, float)), _p(out))
        return out


def erf_kernels(a: float, r: float) -> np.ndarray:
    B = (C.c_double * 4)()
    lib().pgmo_erf_kernels(C.c_double(a), C.c_double(r), B)
    return np.array(B[:])


def bspline(f: float, order: int):
    t, d, s = (C.c_double * order)(), (C.c_double * order)(), (C.c_double * order)()
    lib().pgmo_bspline(C.c_double(f), C.c_int(order), t, d, s)
    return np.array(t[:]), np.array(d[:]), np.array(s[:])
