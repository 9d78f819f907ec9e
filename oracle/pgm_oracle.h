/*
 * pgm_oracle.h -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
 *
 * FP64 CPU restatement of pGM-JAX's per-step polarizable electrostatics (PGMForceField.compute,
 * pgm_jax/md/forcefield.py:2489, with md/pme.py and md/kernels.py).  It is the checker the
 * parity tests compare the CUDA path against, and the timed CPU baseline of bench.py.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 *
 * Units: nm, e, e nm, nm^3, kJ/mol, kJ/mol/nm.  Boxes are lower-triangular with lattice vectors
 * as rows (reduced form, pgm_jax/md/box.py:32).  Atoms of one molecule are contiguous.
 */
#ifndef PGM_ORACLE_H
#define PGM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int n;                 /* atoms */
    int nmol;              /* molecules */
    const int *mol_start;  /* (nmol + 1) first atom of every molecule */
    const double *q;       /* (n) charges [e] */
    const double *radius;  /* (n) Gaussian radii [nm] */
    const double *alpha;   /* (n) polarizabilities [nm^3] */
    const double *rmin_half; /* (n) LJ R* [nm] */
    const double *sqrt_eps;  /* (n) sqrt of the LJ well depth [sqrt(kJ/mol)] */
    const double *mass;    /* (n) masses [amu] */
    int ncov;              /* covalent dipoles */
    const int *cov_i;      /* (ncov) atom carrying the dipole */
    const int *cov_j;      /* (ncov) atom it points to */
    const double *cov_c;   /* (ncov) strength [e nm] */
} pgmo_system;

typedef struct {
    int perm;              /* permanent dipoles (elec "qp" / "qpi") */
    int induce;            /* induced dipoles (elec "qi" / "qpi") */
    int lj;                /* Lennard-Jones rows (vdw "lj") */
    int lj_lrc;            /* long-range LJ correction */
    double cutoff;         /* pair cutoff [nm] */
    double beta;           /* Ewald coefficient [1/nm] */
    int K[3];              /* PME grid */
    int order;             /* B-spline order */
    double tol;            /* max|alpha r| / mean|alpha b| */
    int max_iter;
    int predictor;         /* 0 none, 3 mu3, 4 mu4 */
    int fused;
    int norm_refresh;
    double peek;
    int nthreads;          /* OpenMP threads (0: default) */
    double elec_cutoff;    /* electrostatics cutoff [nm] (0 or >= cutoff: the pair cutoff; forcefield.py:44-58) */
    /* extended-Lagrangian dipoles (forcefield.py:246-282 ExtendedLagrangian, 1452-1650) */
    int iel;               /* 0 none, 1 "0scf", 2 "scf" */
    int iel_order;         /* Niklasson dissipation order K: 0, 3..9 */
    double iel_kappa;      /* NaN: the table's value for K */
    double iel_alpha;      /* NaN: the table's value for K */
    double iel_omega;      /* 0scf: mu = x + omega delta */
    int iel_precond;       /* 0 jacobi, 1 block (molecules of 2..8 atoms) */
    int iel_iter;          /* scf: CG iterations per step (0: to tol) */
    int iel_shadow;        /* 0scf: energy and forces of the shadow potential */
    double local_cut;      /* local preconditioner: cutoff of its short-range rows [nm] (forcefield.py:302-305) */
    int local_niter;       /* its inner CG iterations; 0: Jacobi */
} pgmo_settings;

typedef struct {
    double elec, vdw, total;   /* kJ/mol */
    double virial[9];          /* dE/d eps at fixed mu, minus the tail impulse [kJ/mol] */
    int iterations;
    double residual;
    long long pairs;           /* ordered in-cutoff pairs (both rows) */
} pgmo_result;

/* One force-field step: solve the induced dipoles from the predictor state (mu, hist newest
 * first (4, n, 3), count, norm; updated in place), then energies, forces (n, 3) and virial. */
int pgmo_compute(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H,
                 double *mu, double *hist, int *count, double *norm, double *forces, pgmo_result *res);

/* Energy at fixed induced dipoles mu (PGMForceField.energy_fixed_mu, forcefield.py:2249). */
/* iEL step: as pgmo_compute with the auxiliary dipoles xl (K1, n, 3), K1 = pgmo_iel_len(order),
 * newest first (updated in place); the warm-up steps (count < max(K, 2) + 1) solve to tol. */
int pgmo_compute_iel(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H, double *mu,
                     double *hist, int *count, double *norm, double *xl, double *forces, pgmo_result *res);
int pgmo_iel_len(int order);

int pgmo_energy_fixed_mu(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H,
                         const double *mu, double out[3]);

/* Total field -dU/dd (n, 3) [e/nm^2] of charges q and dipoles d (forcefield.py:1428). */
int pgmo_field(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H,
               const double *q, const double *d, double *field);

/* Permanent dipoles (n, 3) [e nm] (forcefield.py:1032). */
int pgmo_perm_dipoles(const pgmo_system *sys, const double *pos, const double *H, double *p);

/* B_0..B_3 of erf(a r)/r (md/kernels.py:76). */
void pgmo_erf_kernels(double a, double r, double B[4]);

/* B-spline weights and first/second derivatives at offset f (md/pme.py:57). */
void pgmo_bspline(double f, int order, double *theta, double *dtheta, double *d2theta);

#ifdef __cplusplus
}
#endif
#endif
