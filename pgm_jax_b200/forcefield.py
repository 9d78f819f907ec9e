"""PGMForceField on the B200 engine: the call surface of pGM-JAX's force field over the C ABI.

Mirrors pgm_jax/md/forcefield.py: `MDSettings` (flat names of forcefield.py:331-367 for the settings
of this path, `replace` as forcefield.py:458-485), `InductionState` (679-713), `Result` (716-746)
and `PGMForceField` with `compute` (2489), `energy` (2562), `energy_fixed_mu` (2249),
`strain_derivative` (2628), `init_induction` (1436), `rows_for` (2478), `size_rows` / `grow_rows` /
`fit_rows` / `capacity` (1258-1312).  Arrays are torch tensors on the GPU (PyTorch is used only
for device memory and streams); all numerics run in the engine's sm_100a kernels
(csrc/pgm_kernels.cuh).  One instance may hold a batch of systems (replicas, beads, uneven
boxes): their arrays are concatenated and every per-system quantity gains a leading axis.

Units: nm, e, e nm, nm^3, kJ/mol, kJ/mol/nm.
"""

from __future__ import annotations

import ctypes as C
import dataclasses as _dc
from typing import NamedTuple

import math

import numpy as np
import torch

from . import _lib
from .systems import System, grid_size

ELEC_LEVELS = {"q": 0, "qp": 1, "qi": 2, "qpi": 3}
# "mu1": the previous step's dipoles (the plain-CG start the learned guess is measured against);
# "nn": mu4 plus the learned correction (learned.py), mu4 until a model is installed
PREDICTORS = {"none": 0, "mu1": 1, "mu3": 3, "mu4": 4, "nn": 5}

# The settings of MDSettings that this engine implements, with the reference's defaults
# (forcefield.py:142-516).  Other reference settings (IPS, DE / GVDW, the "ls" predictor,
# differentiable solves) are outside this path.
_OUT_OF_SCOPE = {
    "long_range",
    "ips_order", "ips_boundary", "de_alpha", "de_beta", "gvdw_rep",
    "extrap_order", "extrap_steps", "differentiable", "adjoint_tol", "neighbor_list",
}


@_dc.dataclass(frozen=True)
class MDSettings:
    """Force-field and solver settings (flat pmemd-like names of forcefield.py:331-367)."""

    elec: str = "qpi"
    vdw: str = "lj"
    lj_lrc: bool = True
    cutoff: float = 0.9
    elec_cutoff: float | None = None  # < cutoff with vdw "lj": split rows (forcefield.py:44-58)
    skin: float = 0.1
    ewald_beta: float = 4.0
    pme_grid: tuple | None = None
    pme_spacing: float = 0.08
    pme_order: int = 6
    dipole_tol: float = 1e-5
    max_iter: int = 50
    predictor: str = "mu4"
    fused: bool = True
    norm_refresh: int = 1000
    peek: float = 0.65
    # the local preconditioner (Induction.local_cut / local_niter, forcefield.py:302-305): 0 = Jacobi
    local_cut: float = 0.3
    local_niter: int = 0
    precision: str = "mixed"
    # extended-Lagrangian dipoles (ExtendedLagrangian, forcefield.py:246-282)
    iel: str = "none"
    iel_iter: int = 1
    iel_order: int = 7
    iel_kappa: float | None = None
    iel_alpha: float | None = None
    iel_precond: str = "block"
    iel_omega: float = 1.0
    iel_shadow: bool = True

    def replace(self, **changes) -> MDSettings:
        """Return a copy with settings changed (TypeError for unknown names, as forcefield.py:480)."""
        for k in changes:
            if k in _OUT_OF_SCOPE:
                raise ValueError(f"MDSettings: {k!r} is a setting of the reference outside this engine's path")
            if k not in {f.name for f in _dc.fields(self)}:
                raise TypeError(f"MDSettings.replace: unknown setting {k!r}")
        return _dc.replace(self, **changes)

    def __post_init__(self) -> None:
        if self.elec not in ELEC_LEVELS:
            raise ValueError(f"unknown elec {self.elec!r} (q | qp | qi | qpi)")
        if self.vdw not in ("lj", "none"):
            raise ValueError(f"vdw {self.vdw!r}: this engine implements 'lj' and 'none'")
        if self.predictor not in PREDICTORS:
            raise ValueError(f"unknown predictor {self.predictor!r} (mu4 | mu3 | none | nn)")
        if self.precision not in ("mixed", "double"):
            raise ValueError(f"precision {self.precision!r} (mixed | double)")
        if not (self.cutoff > 0):
            raise ValueError("cutoff must be positive")
        if self.elec_cutoff is not None and not (0 < self.elec_cutoff <= self.cutoff):
            raise ValueError("elec_cutoff must be in (0, cutoff] (or None)")
        if self.iel not in ("none", "0scf", "scf"):
            raise ValueError(f"iel {self.iel!r} (none | 0scf | scf)")
        if self.iel_order not in (0, 3, 4, 5, 6, 7, 8, 9):
            raise ValueError("iel_order must be 0 or 3..9")
        if self.iel_precond not in ("block", "jacobi"):
            raise ValueError(f"iel_precond {self.iel_precond!r} (block | jacobi)")
        if not (self.iel_omega > 0) or self.iel_iter < 0:
            raise ValueError("iel_omega must be positive and iel_iter >= 0")
        if not (0 <= self.local_niter <= 8):
            raise ValueError("local_niter must be 0..8")
        if self.local_niter > 0:
            rc = self.elec_cutoff if self.split_rows else self.cutoff
            if not (0 < self.local_cut < rc):
                raise ValueError("local_cut must be positive and below the (electrostatics) cutoff")
            if self.iel != "none":
                raise ValueError("the local preconditioner (local_niter > 0) is not combined with iel")

    @property
    def split_rows(self) -> bool:
        return self.elec_cutoff is not None and self.elec_cutoff < self.cutoff and self.vdw != "none"

    @property
    def has_induction(self) -> bool:
        return "i" in self.elec

    @property
    def perm_dipoles(self) -> bool:
        return "p" in self.elec


# (kappa, a) of Niklasson et al., J. Chem. Phys. 130, 214109 (2009), by dissipation order (the
# defaults when only one of iel_kappa / iel_alpha is given; forcefield.py:667-676)
_XL_TABLE = {0: (1.0, 0.0), 3: (1.69, 0.150), 4: (1.75, 0.057), 5: (1.82, 0.018), 6: (1.84, 0.0055), 7: (1.86, 0.0016),
             8: (1.88, 0.00044), 9: (1.89, 0.00012)}

DSUM_TOL = 3.95e-8  # Amber-convention direct-sum tolerance of the default pair 0.9 nm / 4.0 nm^-1


def ewald_beta_for(elec_cutoff: float, dsum_tol: float = DSUM_TOL) -> float:
    """Ewald coefficient [1/nm] with erfc(beta rc) / rc_A = dsum_tol, rc_A the cutoff in Angstrom,
    by bisection (forcefield.py:523-567): 0.9 nm -> 4.0, 0.7 nm -> 5.19 nm^-1."""
    rc = float(elec_cutoff)
    if not rc > 0.0:
        raise ValueError(f"elec_cutoff must be positive, got {elec_cutoff}")
    f = lambda b: math.erfc(b * rc) / (10.0 * rc) - dsum_tol  # noqa: E731
    if not (dsum_tol > 0.0 and f(0.0) > 0.0):
        raise ValueError(f"dsum_tol must be in (0, 1/rc_A) = (0, {1.0 / (10.0 * rc):.3g}), got {dsum_tol}")
    lo, hi = 0.0, 1.0
    while f(hi) > 0.0:
        hi *= 2.0
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0.0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def elec_cutoff_settings(elec_cutoff: float, dsum_tol: float = DSUM_TOL, exponent: float = 1.6) -> dict:
    """MDSettings arguments for a shorter electrostatics cutoff (forcefield.py:570-601): the Ewald
    coefficient for it and the PME spacing 0.08 nm (4.0 / beta)^exponent."""
    b = ewald_beta_for(elec_cutoff, dsum_tol)
    return {"elec_cutoff": float(elec_cutoff), "ewald_beta": b, "pme_spacing": 0.08 * (4.0 / b) ** exponent}


@_dc.dataclass
class InductionState:
    """Induced-dipole solver state (forcefield.py:679-713); per-system scalars have shape (n_systems,)."""

    mu: torch.Tensor     # (N, 3) float64
    hist: torch.Tensor   # (4, N, 3) float64, newest first
    count: torch.Tensor  # (S,) int32
    norm: torch.Tensor   # (S,) float64
    xl: torch.Tensor | None = None  # iEL: (pgm_iel_len(order), N, 3) float64 auxiliary dipoles, newest first

    def clone(self) -> InductionState:
        return InductionState(self.mu.clone(), self.hist.clone(), self.count.clone(), self.norm.clone(),
                              None if self.xl is None else self.xl.clone())

    def _c(self):
        return _lib.PgmInduction(self.mu.data_ptr(), self.hist.data_ptr(), self.count.data_ptr(), self.norm.data_ptr(),
                                 None if self.xl is None else self.xl.data_ptr())


class Result(NamedTuple):
    """Result of compute (forcefield.py:716-746) plus the molecular virial of the step."""

    energy: dict          # "elec", "vdw", "total": (S,) float64 [kJ/mol]
    forces: torch.Tensor  # (N, 3) float64 [kJ/mol/nm]
    induction: InductionState
    iterations: torch.Tensor  # (S,) int32
    residual: torch.Tensor    # (S,) float64
    overflow: torch.Tensor    # (S,) bool
    virial: torch.Tensor      # (S, 3, 3) float64 [kJ/mol]
    status: torch.Tensor      # (S,) int32 (PGM_STATUS_* bits)


def _ptr(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def _f64(x, dev) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=dev)


class PGMForceField:
    """The pGM + LJ force field of one system or a batch of systems (forcefield.py:810-2695).

        ff = PGMForceField(system, H, MDSettings())
        res = ff.compute(pos, H, None, ff.init_induction())
        res.energy["total"], res.forces, res.virial

    `system`, `H` may be lists (a batch: replicas, beads, uneven boxes); `pme_grids` then gives one
    grid per system (default: from pme_grid or pme_spacing and each box).
    """

    def __init__(self, system, H, settings: MDSettings = MDSettings(), row_capacity: int | None = None, device: int = 0,
                 pme_grids=None, elec_capacity: int | None = None) -> None:
        if elec_capacity is not None and not settings.split_rows:
            raise ValueError("elec_capacity applies only to split rows (elec_cutoff < cutoff with a van der Waals term)")
        self.systems = list(system) if isinstance(system, (list, tuple)) else [system]
        boxes = [np.asarray(h, float) for h in H] if isinstance(H, (list, tuple)) else [np.asarray(H, float)] * len(self.systems)
        if len(boxes) != len(self.systems):
            raise ValueError("one box per system")
        self.s = settings
        self.device = torch.device("cuda", device)
        self.nsys = len(self.systems)
        self.n = sum(s.n for s in self.systems)
        if pme_grids is None:
            pme_grids = [tuple(settings.pme_grid) if settings.pme_grid else grid_size(b, settings.pme_spacing) for b in boxes]
        self.grids = [tuple(int(k) for k in g) for g in pme_grids]
        self.offsets = np.cumsum([0] + [s.n for s in self.systems])
        lib = _lib.load()
        st = _lib.PgmSettings(
            ELEC_LEVELS[settings.elec], int(settings.vdw == "lj"), int(settings.lj_lrc),
            int(settings.precision == "double"), float(settings.cutoff), float(settings.ewald_beta), int(settings.pme_order),
            float(settings.dipole_tol), int(settings.max_iter), PREDICTORS[settings.predictor], int(settings.fused),
            int(settings.norm_refresh), float(settings.peek), int(row_capacity or 0), float(settings.skin), 0,
            float(settings.elec_cutoff or 0.0), int(elec_capacity or 0),
            {"none": 0, "0scf": 1, "scf": 2}[settings.iel], int(settings.iel_order),
            int(settings.iel_kappa is not None or settings.iel_alpha is not None),
            float(settings.iel_kappa if settings.iel_kappa is not None else _XL_TABLE[settings.iel_order][0]),
            float(settings.iel_alpha if settings.iel_alpha is not None else _XL_TABLE[settings.iel_order][1]),
            float(settings.iel_omega), 0 if settings.iel_precond == "block" else 1, int(settings.iel_iter),
            int(not settings.iel_shadow), float(settings.local_cut), int(settings.local_niter),
        )
        descs = (_lib.PgmSystemDesc * self.nsys)()
        self._keep = []
        for k, (sy, b, g) in enumerate(zip(self.systems, boxes, self.grids)):
            d = descs[k]
            d.n_atoms, d.n_mol = sy.n, sy.nmol
            d.mol_start = self._arr(sy.mol_start, np.int32, _lib._pi)
            d.q = self._arr(sy.q, np.float64, _lib._pd)
            d.radius = self._arr(sy.radius, np.float64, _lib._pd)
            d.alpha = self._arr(sy.alpha, np.float64, _lib._pd)
            d.lj_rmin_half = self._arr(sy.lj_rmin_half, np.float64, _lib._pd)
            d.lj_sqrt_eps = self._arr(sy.lj_sqrt_eps, np.float64, _lib._pd)
            d.masses = self._arr(sy.masses, np.float64, _lib._pd)
            d.n_cov = len(sy.cov_i)
            d.cov_i = self._arr(sy.cov_i, np.int32, _lib._pi)
            d.cov_j = self._arr(sy.cov_j, np.int32, _lib._pi)
            d.cov_c = self._arr(sy.cov_c, np.float64, _lib._pd)
            d.pme_grid[:] = list(g)
            d.box0[:] = list(b.reshape(-1))
        h = C.c_void_p()
        torch.cuda.init()
        _lib.check(lib.pgm_create(C.byref(st), descs, self.nsys, device, C.byref(h)))
        self._h = h
        self._lib = lib
        self._keep = []
        dev = self.device
        S = self.nsys
        self._energy = torch.zeros((S, 3), dtype=torch.float64, device=dev)
        self._virial = torch.zeros((S, 3, 3), dtype=torch.float64, device=dev)
        self._iters = torch.zeros(S, dtype=torch.int32, device=dev)
        self._resid = torch.zeros(S, dtype=torch.float64, device=dev)
        self._status = torch.zeros(S, dtype=torch.int32, device=dev)

    def _arr(self, x, dt, ptype):
        a = np.ascontiguousarray(x, dtype=dt)
        self._keep.append(a)
        return a.ctypes.data_as(ptype)

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.pgm_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------------ state and sizes
    def init_induction(self) -> InductionState:
        """A fresh solver state: zero dipoles and history, normaliser 1 (forcefield.py:1436-1450)."""
        dev = self.device
        xl = None
        if self.s.iel != "none":
            xl = torch.zeros((self._lib.pgm_iel_len(int(self.s.iel_order)), self.n, 3), dtype=torch.float64, device=dev)
        return InductionState(
            torch.zeros((self.n, 3), dtype=torch.float64, device=dev),
            torch.zeros((4, self.n, 3), dtype=torch.float64, device=dev),
            torch.zeros(self.nsys, dtype=torch.int32, device=dev),
            torch.ones(self.nsys, dtype=torch.float64, device=dev),
            xl,
        )

    @property
    def capacity(self) -> int:
        """Pairs kept per row."""
        return int(self._lib.pgm_row_capacity(self._h))

    def set_capacity(self, mc: int) -> None:
        _lib.check(self._lib.pgm_set_row_capacity(self._h, int(mc)))

    @property
    def elec_capacity(self) -> int:
        """Split rows: electrostatic pairs kept per row (else the row capacity)."""
        return int(self._lib.pgm_elec_capacity(self._h))

    def set_elec_capacity(self, c: int) -> None:
        _lib.check(self._lib.pgm_set_elec_capacity(self._h, int(c)))

    def size_rows(self, pos, H, idx=None, factor: float = 1.2) -> int:
        """Set the capacity from the largest row at pos, with half the head-room `factor` gives (forcefield.py:1269);
        with split rows both parts."""
        grow = lambda c: int(np.ceil((c * (1.0 + 0.5 * (factor - 1.0)) + 8) / 8.0) * 8)  # noqa: E731
        self.set_capacity(max(self.capacity, 1024))
        if self.s.split_rows:
            self.set_elec_capacity(max(self.elec_capacity, 512))
        self.compute(pos, H, idx, self.init_induction())
        c = int(self._lib.pgm_max_row_count(self._h))
        if self.s.split_rows:
            v = int(self._lib.pgm_max_vdw_count(self._h))
            self.set_elec_capacity(grow(c))
            self.set_capacity(self.elec_capacity + grow(v))
        else:
            self.set_capacity(grow(c))
        return self.capacity

    @property
    def list_capacity(self) -> int:
        """Candidates kept per atom in the engine's Verlet list."""
        return int(self._lib.pgm_list_capacity(self._h))

    def set_list_capacity(self, c: int) -> None:
        _lib.check(self._lib.pgm_set_list_capacity(self._h, int(c)))

    def list_rebuilds(self) -> int:
        """How many times the Verlet candidate list has been rebuilt."""
        return int(self._lib.pgm_list_rebuilds(self._h))

    def grow_rows(self, old: int) -> None:
        """Widen the rows by at least 8 after an overflow at capacity `old` (forcefield.py:1286); with
        split rows each part to the largest count of the last build + 8."""
        if self.s.split_rows:
            e, v = int(self._lib.pgm_max_row_count(self._h)), int(self._lib.pgm_max_vdw_count(self._h))
            self.set_elec_capacity(max(self.elec_capacity, e + 8))
            self.set_capacity(max(self.capacity, self.elec_capacity + v + 8, int(old) + 8))
            return
        self.set_capacity(max(self.capacity, int(old) + 8))

    def fit_rows(self, caps) -> None:
        """Set a capacity that fits every one of `caps` (forcefield.py:1298)."""
        caps = [c for c in caps if c]
        if caps:
            self.set_capacity(max(caps))

    def rows_for(self, pos, H) -> np.ndarray:
        """Candidate rows (N, C) of every atom within the cutoff, padding N (host; forcefield.py:2478)."""
        out = []
        for k, sy in enumerate(self.systems):
            x = np.asarray(pos, float)[self.offsets[k]:self.offsets[k + 1]]
            h = np.asarray(H, float)
            h = h[k] if h.ndim == 3 else h
            d = x[:, None, :] - x[None, :, :]
            for c in (2, 1, 0):
                n = np.round(d[..., c] / h[c, c])
                d = d - n[..., None] * h[c][None, None, :]
            r2 = (d * d).sum(-1)
            np.fill_diagonal(r2, np.inf)
            rows = [np.nonzero(r2[i] < self.s.cutoff**2)[0] for i in range(sy.n)]
            w = max(len(r) for r in rows)
            a = np.full((sy.n, w), sy.n, np.int32)
            for i, r in enumerate(rows):
                a[i, : len(r)] = r
            out.append(a)
        w = max(a.shape[1] for a in out)
        return np.concatenate([np.pad(a, ((0, 0), (0, w - a.shape[1])), constant_values=a.shape[0]) for a in out])

    # ------------------------------------------------------------------ calls
    def _boxes(self, H) -> torch.Tensor:
        b = _f64(H, self.device)
        if b.ndim == 2:
            b = b.expand(self.nsys, 3, 3).contiguous()
        return b

    def _idx(self, idx):
        if idx is None:
            return None, 0
        t = torch.as_tensor(np.asarray(idx, np.int32) if not isinstance(idx, torch.Tensor) else idx, device=self.device)
        t = t.to(torch.int32).contiguous()
        return t, int(t.shape[1])

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def compute(self, pos, H, idx=None, ind: InductionState | None = None) -> Result:
        """Solve the induced dipoles (predicted guess), then energies, forces and virial (forcefield.py:2489).

        `ind` is updated in place (mu, history, count, norm) and returned in the Result.
        """
        ind = self.init_induction() if ind is None else ind
        x = _f64(pos, self.device)
        b = self._boxes(H)
        it, w = self._idx(idx)
        F = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        di = ind._c()
        E, V, I, R, Sst = self._energy.clone(), self._virial.clone(), self._iters.clone(), self._resid.clone(), self._status.clone()
        out = _lib.PgmOutputs(E.data_ptr(), F.data_ptr(), V.data_ptr(), I.data_ptr(), R.data_ptr(), Sst.data_ptr())
        _lib.check(self._lib.pgm_compute(self._h, self._stream(), _ptr(x), _ptr(b), _ptr(it), w, C.byref(di), C.byref(out)))
        energy = {"elec": E[:, 0], "vdw": E[:, 1], "total": E[:, 2]}
        return Result(energy, F, ind, I, R, (Sst & (_lib.STATUS_ROW_OVERFLOW | _lib.STATUS_LIST_OVERFLOW)) != 0, V, Sst)

    def compute_into(self, pos: torch.Tensor, boxes: torch.Tensor, ind: InductionState, forces: torch.Tensor) -> Result:
        """compute() into persistent buffers, with no allocation (for CUDA-graph capture).

        pos (N, 3) and boxes (S, 3, 3) float64 CUDA tensors; forces (N, 3) receives the forces.  The
        energy, virial, iterations, residual and status of the Result are this instance's buffers,
        overwritten by the next call.
        """
        di = ind._c()
        out = _lib.PgmOutputs(self._energy.data_ptr(), forces.data_ptr(), self._virial.data_ptr(), self._iters.data_ptr(),
                              self._resid.data_ptr(), self._status.data_ptr())
        _lib.check(self._lib.pgm_compute(self._h, self._stream(), _ptr(pos), _ptr(boxes), None, 0, C.byref(di), C.byref(out)))
        E = self._energy
        return Result({"elec": E[:, 0], "vdw": E[:, 1], "total": E[:, 2]}, forces, ind, self._iters, self._resid,
                      (self._status & (_lib.STATUS_ROW_OVERFLOW | _lib.STATUS_LIST_OVERFLOW)) != 0, self._virial, self._status)

    def energy(self, pos, H, idx=None, ind: InductionState | None = None):
        """Energy only, dipoles solved from ind.mu, no history push (forcefield.py:2562).

        Returns (E_total (S,), ind with the converged mu, iterations (S,), overflow (S,)).
        """
        ind = self.init_induction() if ind is None else ind.clone()
        x = _f64(pos, self.device)
        b = self._boxes(H)
        it, w = self._idx(idx)
        di = ind._c()
        E, I, Sst = self._energy.clone(), self._iters.clone(), self._status.clone()
        _lib.check(self._lib.pgm_energy(self._h, self._stream(), _ptr(x), _ptr(b), _ptr(it), w, C.byref(di), _ptr(E), _ptr(I),
                                        _ptr(Sst)))
        return E[:, 2], ind, I, (Sst & _lib.STATUS_ROW_OVERFLOW) != 0

    def energy_fixed_mu(self, pos, H, mu, idx=None):
        """Total energy and parts with the induced dipoles held at mu (forcefield.py:2249); also forces, virial."""
        x = _f64(pos, self.device)
        b = self._boxes(H)
        m = _f64(mu, self.device)
        it, w = self._idx(idx)
        E, V = self._energy.clone(), self._virial.clone()
        F = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        _lib.check(self._lib.pgm_energy_fixed_mu(self._h, self._stream(), _ptr(x), _ptr(b), _ptr(it), w, _ptr(m), _ptr(E), _ptr(F),
                                                 _ptr(V), None))
        return E[:, 2], {"elec": E[:, 0], "vdw": E[:, 1], "forces": F, "virial": V}

    def strain_derivative(self, pos, H, idx, mu) -> torch.Tensor:
        """dE/d eps (S, 3, 3) at fixed mu with molecular scaling, minus the tail impulse (forcefield.py:2628)."""
        return self.energy_fixed_mu(pos, H, mu, idx)[1]["virial"]

    def field(self, pos, H, d, charges: bool = True) -> torch.Tensor:
        """The total field -dU/dd (N, 3) [e/nm^2] of the charges (if `charges`) and dipoles d (forcefield.py:1428)."""
        x = _f64(pos, self.device)
        b = self._boxes(H)
        dd = _f64(d, self.device)
        out = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        _lib.check(self._lib.pgm_field(self._h, self._stream(), _ptr(x), _ptr(b), int(charges), _ptr(dd), _ptr(out)))
        return out

    def last_launch_count(self) -> int:
        """Kernels launched by the last call."""
        return int(self._lib.pgm_last_launch_count(self._h))

    def set_nn_fallback(self, factor: float) -> None:
        """Learned guess (predictor "nn"): restart a solve from the mu4 extrapolation when the start
        residual of the learned guess is above `factor` times the recorded mean of the extrapolation's
        (0: never; default 2)."""
        _lib.check(self._lib.pgm_set_nn_fallback(self._h, float(factor)))

    def nn_fallback_stats(self) -> dict:
        """Per system: fallbacks so far and the recorded mean start residual of the extrapolation."""
        fb = np.zeros(self.nsys, np.int64)
        ref = np.zeros(self.nsys)
        _lib.check(self._lib.pgm_nn_fallback_stats(self._h, C.c_void_p(fb.ctypes.data), C.c_void_p(ref.ctypes.data)))
        return {"fallbacks": fb, "ref_err": ref}

    def tuning(self) -> dict:
        """The kernel variants in use and the autotuner's timings (pgm_tuning)."""
        t = _lib.PgmTuning()
        _lib.check(self._lib.pgm_tuning(self._h, C.byref(t)))
        return {"rowfield_lanes": t.rowfield_lanes, "forces_blocks_per_sm": t.forces_blocks_per_sm,
                "sweep_early": t.sweep_early, "rowfield_grid": t.rowfield_grid, "rowfield_ms": list(t.rowfield_ms),
                "forces_ms": list(t.forces_ms), "sweep_ms": list(t.sweep_ms), "grid_ms": list(t.grid_ms),
                "tuned": bool(t.tuned), "from_cache": bool(t.from_cache)}

    def set_tuning(self, rowfield_lanes: int = 0, forces_blocks_per_sm: int = 0, sweep_early: int = -1,
                   rowfield_grid: int = -1) -> None:
        """Fix the kernel variants (0 / -1 keeps one; all so: autotune again at the next direct step)."""
        _lib.check(self._lib.pgm_set_tuning(self._h, int(rowfield_lanes), int(forces_blocks_per_sm), int(sweep_early),
                                            int(rowfield_grid)))

    def autotune(self) -> dict:
        """Time the kernel variants now on the last step's rows; returns tuning()."""
        _lib.check(self._lib.pgm_autotune(self._h, self._stream()))
        return self.tuning()
