"""Molecule templates, systems and the synthetic boxes used by tests and benchmarks.

A `Molecule` carries per-atom pGM parameters (charges, Gaussian radii, polarizabilities, covalent
dipoles, Lennard-Jones R* and sqrt(eps), masses), in the reference's internal units (nm, e, e nm,
nm^3, sqrt(kJ/mol), amu; pgm_jax/system.py:117-215).  A `System` concatenates molecules, atoms of a
molecule contiguous (pgm_jax/system.py:500-530).

Builders:
  * `pgm3p25_water`: the pGM3P-25 rigid water, numbers taken from the POL_GAUSS_* and LJ sections of
    the reference's examples/water512/pgm3p25_512.prmtop (read by pgm_jax/param.py:113, converted
    as param.py:237-248 and param.py:281-307 do).
  * `toy_water`, `toy_methanol`, `small_box`: restatements of pgm_jax/models/toy.py:26-77,143-183
    (the 114-atom triclinic water/methanol box of the reference's regression harness), so that its
    golden single point can be reproduced from the same numpy seed.
  * `water_box`: n^3 randomly oriented rigid waters on a jittered cubic lattice (the synthetic
    benchmark boxes), with the orientation draw of pgm_jax/models/toy.py:107-141.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

ANG_NM = 0.1
KCAL = 4.184
MASSES = {"H": 1.008, "C": 12.011, "O": 15.999}  # pgm_jax/system.py:96-108


@dataclass
class Molecule:
    """One molecule template (per-atom arrays of length m; cov entries (i, j, c) local indices)."""

    name: str
    elements: list
    q: np.ndarray
    radius: np.ndarray
    alpha: np.ndarray
    cov: list = field(default_factory=list)
    lj_rmin_half: np.ndarray | None = None
    lj_sqrt_eps: np.ndarray | None = None
    masses: np.ndarray | None = None

    def __post_init__(self) -> None:
        m = len(self.elements)
        self.q = np.asarray(self.q, float).reshape(m)
        self.radius = np.asarray(self.radius, float).reshape(m)
        self.alpha = np.asarray(self.alpha, float).reshape(m)
        self.lj_rmin_half = np.zeros(m) if self.lj_rmin_half is None else np.asarray(self.lj_rmin_half, float)
        self.lj_sqrt_eps = np.zeros(m) if self.lj_sqrt_eps is None else np.asarray(self.lj_sqrt_eps, float)
        if self.masses is None:
            self.masses = np.array([MASSES[e] for e in self.elements])
        self.masses = np.asarray(self.masses, float)

    @property
    def n(self) -> int:
        return len(self.elements)


class System:
    """Molecules concatenated into flat per-atom arrays (float64 / int32)."""

    def __init__(self, molecules: list[Molecule]) -> None:
        self.molecules = list(molecules)
        offs = np.cumsum([0] + [m.n for m in molecules])
        self.mol_start = offs.astype(np.int32)
        self.n = int(offs[-1])
        self.nmol = len(molecules)
        self.mol = np.concatenate([np.full(m.n, k, np.int32) for k, m in enumerate(molecules)])
        cat = lambda name: np.concatenate([getattr(m, name) for m in molecules]).astype(float)  # noqa: E731
        self.q = cat("q")
        self.radius = cat("radius")
        self.alpha = cat("alpha")
        self.lj_rmin_half = cat("lj_rmin_half")
        self.lj_sqrt_eps = cat("lj_sqrt_eps")
        self.masses = cat("masses")
        ci, cj, cc = [], [], []
        for k, m in enumerate(molecules):
            for i, j, c in m.cov:
                ci.append(offs[k] + i)
                cj.append(offs[k] + j)
                cc.append(c)
        self.cov_i = np.array(ci, np.int32)
        self.cov_j = np.array(cj, np.int32)
        self.cov_c = np.array(cc, float)


# ----------------------------------------------------------------------------- pGM3P-25 water
def pgm3p25_water() -> Molecule:
    """Return the pGM3P-25 rigid water (O, H1, H2).

    prmtop values: monopoles -2.04056220 / +1.02028110 e, radii 0.605150752 / 0.536231183 A,
    polarizabilities 1.11765163 / 0.329630770 A^3, covalent dipoles O->H -0.191201350 e A and
    H->O +0.0858770326 e A, LJ A = 5.81935564e5 kcal A^12/mol, B = 5.94825035e2 kcal A^6/mol on O,
    masses 16.00 / 1.008.
    """
    A, B = 5.81935564e5, 5.94825035e2
    rmin = (2.0 * A / B) ** (1.0 / 6.0)  # A
    eps = B * B / (4.0 * A)  # kcal/mol
    c_oh, c_ho = -0.191201350 * ANG_NM, 0.0858770326 * ANG_NM
    return Molecule(
        "WAT",
        ["O", "H", "H"],
        np.array([-2.04056220, 1.02028110, 1.02028110]),
        np.array([0.605150752, 0.536231183, 0.536231183]) * ANG_NM,
        np.array([1.11765163, 0.329630770, 0.329630770]) * ANG_NM**3,
        cov=[(0, 1, c_oh), (0, 2, c_oh), (1, 0, c_ho), (2, 0, c_ho)],
        lj_rmin_half=np.array([rmin / 2.0 * ANG_NM, 0.0, 0.0]),
        lj_sqrt_eps=np.array([math.sqrt(eps * KCAL), 0.0, 0.0]),
        masses=np.array([16.0, 1.008, 1.008]),
    )


def water_geometry(r: float = 0.09572, theta_deg: float = 104.52) -> np.ndarray:
    """O, H, H (3, 3) [nm]: O at the origin, bisector along +y, in the xy plane (toy.py:80-87)."""
    t = np.radians(theta_deg / 2)
    return np.array([[0, 0, 0], [r * np.sin(t), r * np.cos(t), 0], [-r * np.sin(t), r * np.cos(t), 0]])


def water_box(n_side: int, edge_nm: float, seed: int = 0, jitter: float = 0.01, mol: Molecule | None = None,
              n_water: int | None = None):
    """Return (System, positions (3 n^3, 3) [nm], box (3, 3) [nm]) of a jittered lattice of waters.

    Orientations are the Q factor of a Gaussian 3x3 matrix from np.random.default_rng(seed), as in
    toy.water_lattice (toy.py:107-141); each molecule is centred on its cell centre plus Gaussian
    jitter of `jitter` nm (as toy.small_box, toy.py:173).  n_water < n^3: that many sites of the
    lattice, chosen at random (seeded), the others left empty.
    """
    rng = np.random.default_rng(seed)
    w = water_geometry()
    w = w - w.mean(0)
    sp = edge_nm / n_side
    pos = []
    for i in range(n_side):
        for j in range(n_side):
            for k in range(n_side):
                Q = np.linalg.qr(rng.normal(size=(3, 3)))[0]
                c = (np.array([i, j, k]) + 0.5) * sp + rng.normal(scale=jitter, size=3)
                pos.append(w @ Q.T + c)
    nw = n_side**3
    if n_water is not None and n_water < nw:
        keep = np.sort(rng.choice(nw, size=n_water, replace=False))
        pos = [pos[k] for k in keep]
        nw = n_water
    m = pgm3p25_water() if mol is None else mol
    return System([m] * nw), np.concatenate(pos), np.eye(3) * edge_nm


# ----------------------------------------------------------------------------- toy systems
def toy_water() -> Molecule:
    """The toy water template of toy.py:26-44."""
    return Molecule(
        "WAT",
        ["O", "H", "H"],
        np.array([-0.8, 0.4, 0.4]),
        np.array([0.06, 0.05, 0.05]),
        np.array([1.0e-3, 0.3e-3, 0.3e-3]),
        cov=[(0, 1, -0.02), (0, 2, -0.02), (1, 0, 0.008), (2, 0, 0.008)],
        lj_rmin_half=[0.178, 0.0, 0.0],
        lj_sqrt_eps=[0.80, 0.0, 0.0],
    )


def toy_methanol() -> tuple[Molecule, np.ndarray]:
    """The toy methanol template and its geometry [nm] (toy.py:47-77)."""
    x = (
        np.array(
            [
                [-0.0467, 0.6590, 0.0],
                [-0.0467, -0.7598, 0.0],
                [-1.0830, 0.9930, 0.0],
                [0.4406, 1.0735, 0.8902],
                [0.4406, 1.0735, -0.8902],
                [0.8785, -1.0591, 0.0],
            ]
        )
        * 0.1
    )
    m = Molecule(
        "MeOH",
        ["C", "O", "H", "H", "H", "H"],
        np.array([0.12, -0.62, 0.02, 0.02, 0.02, 0.44]),
        np.array([0.07, 0.06, 0.05, 0.05, 0.05, 0.05]),
        np.array([1.2e-3, 0.8e-3, 0.4e-3, 0.4e-3, 0.4e-3, 0.3e-3]),
        cov=[(0, 1, 0.01), (1, 0, -0.01), (1, 5, -0.02), (5, 1, 0.005)]
        + [c for h in (2, 3, 4) for c in ((0, h, 0.002), (h, 0, -0.002))],
        lj_rmin_half=[0.19, 0.172, 0.139, 0.139, 0.139, 0.02],
        lj_sqrt_eps=[0.33, 0.85, 0.20, 0.20, 0.20, 0.1],
    )
    return m, x


def reduce_box(H: np.ndarray) -> np.ndarray:
    """Reduced lower-triangular box (pgm_jax/md/box.py:32-59)."""
    H = np.array(H, float)
    a, b, c = H
    c = c - b * np.round(c[1] / b[1])
    c = c - a * np.round(c[0] / a[0])
    b = b - a * np.round(b[0] / a[0])
    return np.array([a, b, c])


def small_box(seed: int = 0, nw: int = 30, nm: int = 4):
    """Waters and methanols on a jittered lattice in a skewed triclinic box (toy.py:143-183).

    Returns (System, positions (N, 3) [nm], box (3, 3) [nm]); methanols first, then waters.
    """
    rng = np.random.default_rng(seed)
    H = reduce_box(np.array([[1.75, 0.0, 0.0], [0.45, 1.70, 0.0], [-0.40, 0.50, 1.65]]))
    w = water_geometry()
    m, xm = toy_methanol()
    xm = xm - xm.mean(0)
    W = toy_water()
    mols, pos = [], []
    grid = np.array([[i, j, k] for i in range(4) for j in range(4) for k in range(3)], float)
    grid = (grid + 0.5) / np.array([4, 4, 3])
    for n, f in enumerate(grid[rng.permutation(len(grid))][: nw + nm]):
        R = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        c = f @ H + rng.normal(scale=0.01, size=3)
        if n < nm:
            mols.append(m)
            pos.append(xm @ R.T + c)
        else:
            mols.append(W)
            pos.append((w - w.mean(0)) @ R.T + c)
    return System(mols), np.concatenate(pos), H


def grid_size(H: np.ndarray, spacing: float = 0.08, factors=(2, 3, 5)) -> tuple[int, int, int]:
    """Smallest even FFT-friendly grid with at most `spacing` between lattice planes (pme.py:134-172)."""
    H = np.asarray(H, float)
    V = abs(np.linalg.det(H))
    heights = [
        V / np.linalg.norm(np.cross(H[1], H[2])),
        V / np.linalg.norm(np.cross(H[2], H[0])),
        V / np.linalg.norm(np.cross(H[0], H[1])),
    ]

    def ok(n: int) -> bool:
        for f in factors:
            while n % f == 0:
                n //= f
        return n == 1

    out = []
    for h in heights:
        n = max(8, int(np.ceil(h / spacing)))
        while not ok(n) or n % 2:
            n += 1
        out.append(n)
    return tuple(out)
