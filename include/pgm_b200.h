/*
 * pgm_b200.h -- C ABI of the B200 (sm_100a) pGM electrostatics engine.
 *
 * One handle holds one force field over a batch of independent periodic systems (one system, or
 * REMD replicas, PIMD beads, boxes of uneven sizes), each with its own box and PME mesh, evaluated
 * together by the same kernels.  All array arguments of the compute calls are DEVICE pointers
 * owned by the caller (as the buffers of a jax.ffi custom call are), concatenated over the systems
 * in system order; the *_host variants take host pointers and copy.
 *
 * Units: nm, e, e nm, nm^3, kJ/mol, kJ/mol/nm (pgm_jax/md/forcefield.py:100).  Boxes are
 * lower-triangular, lattice vectors as rows, in reduced form (pgm_jax/md/box.py:32).
 *
 * Graphs: pgm_compute and pgm_energy may be called while the stream is being captured (stream
 * capture, any mode); the CG loop is then recorded as a device-side while loop (conditional graph
 * node) that runs until every system has converged or reached max_iter, so a replayed step never
 * returns to the host.  Outside capture the loop is driven from the host.
 *
 * Errors: every entry point returns a PgmStatus; nothing is thrown across the boundary.
 * Per-system conditions of a step (row overflow, CG not converged, non-finite energy) come back in
 * the `status` output word of each system, as the reference reports them in Result.overflow and
 * Result.residual (forcefield.py:716-746) and its driver checks for non-finite energies.
 */
#ifndef PGM_B200_H
#define PGM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PGM_OK = 0,
    PGM_ERR_INVALID = 1,   /* bad argument or setting (ValueError at construction, forcefield.py:902-906) */
    PGM_ERR_CUDA = 2,      /* a CUDA runtime error; pgm_last_error() has the text */
    PGM_ERR_NO_DEVICE = 3,
    PGM_ERR_UNSUPPORTED = 4
} PgmStatus;

/* Bits of the per-system status word of a step. */
#define PGM_STATUS_ROW_OVERFLOW 0x1u   /* a row had more in-cutoff pairs than the capacity: results invalid, resize and repeat */
#define PGM_STATUS_CG_MAXITER   0x2u   /* CG stopped at max_iter above the tolerance */
#define PGM_STATUS_NONFINITE    0x4u   /* non-finite energy */
#define PGM_STATUS_BAD_BOX      0x8u   /* box not lower triangular / too small for the cutoff */
#define PGM_STATUS_LIST_OVERFLOW 0x10u /* an atom had more candidates within cutoff + skin than the list capacity */
#define PGM_STATUS_SHORT_OVERFLOW 0x20u /* local preconditioner: an atom had more than 48 entries inside local_cut;
                                          the first 48 were used (results valid, iterations may differ) */

/* Settings of one handle: the MDSettings fields of the path (forcefield.py:386-516). */
typedef struct {
    int elec;           /* 0 "q", 1 "qp", 2 "qi", 3 "qpi" (options.py ELEC_LEVELS) */
    int vdw;            /* 0 "none", 1 "lj" */
    int lj_lrc;         /* Amber vdwmeth=1 tail (lj.py:87) */
    int precision;      /* 0 "mixed" (FP32 kernels, FP64 reductions), 1 "double" */
    double cutoff;      /* pair cutoff [nm] (Cutoffs.cutoff) */
    double ewald_beta;  /* [1/nm] (PMESettings.ewald_beta) */
    int pme_order;      /* 4, 6 or 8 (PMESettings.order) */
    double dipole_tol;  /* max|alpha r| / mean|alpha b| (Induction.tol) */
    int max_iter;       /* Induction.max_iter */
    int predictor;      /* 0 "none", 3 "mu3", 4 "mu4" (Induction.predictor); 1 the previous step's
                           dipoles; 5 mu4 + the learned correction (pgm_set_nn_model; mu4 until
                           a model is set) */
    int fused;          /* Induction.fused */
    int norm_refresh;   /* Induction.norm_refresh */
    double peek;        /* Induction.peek */
    int row_capacity;   /* pairs kept per row; 0: sized from the density (PGMForceField.size_rows) */
    double skin;        /* Verlet skin of the engine's candidate list [nm] (NeighborList.skin); clipped so
                           that cutoff + skin fits the smallest box, 0: rebuilt every step */
    int list_capacity;  /* candidates kept per atom; 0: sized from the density */
    double elec_cutoff; /* electrostatics cutoff [nm] (Cutoffs.elec_cutoff); 0 or = cutoff: one cutoff.
                           Below cutoff (with vdw "lj") the rows are split (forcefield.py:44-58,
                           1197-1238): [0, elec_capacity) pairs inside elec_cutoff, then the pairs
                           between elec_cutoff and cutoff with a nonzero LJ term; the field sweeps
                           stream the first part only.  ewald_beta and the mesh must suit it. */
    int elec_capacity;  /* split rows: electrostatic pairs kept per row (0: from the density) */
    /* Extended-Lagrangian induced dipoles (Induction.iel, forcefield.py:246-282, 1452-1650): the
       auxiliary dipoles PgmInduction.xl follow Niklasson's dissipative Verlet
       x_{n+1} = 2 x_n - x_{n-1} + kappa (mu_n - x_n) + a sum_k c_k x_{n-k}; the first
       max(order, 2) + 1 steps solve to dipole_tol, later ones start from x = xl[0]. */
    int iel;            /* 0 "none" (the predictor + CG above), 1 "0scf" (mu = x + omega delta, delta =
                           alpha r(x) or M^-1 r(x), one field sweep, no CG), 2 "scf" (iel_iter CG
                           iterations from x; 0: to dipole_tol) */
    int iel_order;      /* dissipation order K: 0 or 3..9 (the reference's default is 7) */
    int iel_custom;     /* 1: iel_kappa and iel_alpha below; 0: Niklasson's values for the order */
    double iel_kappa;   /* kappa = (omega dt)^2 of the auxiliary dipoles' harmonic coupling */
    double iel_alpha;   /* dissipation strength a */
    double iel_omega;   /* 0scf: mu = x + omega delta (0 is read as 1) */
    int iel_precond;    /* 0scf: 0 "block" (M = 1/alpha + the rows inside molecules of 2..8 atoms),
                           1 "jacobi" (delta = alpha r) */
    int iel_iter;       /* scf: CG iterations per step (0: to dipole_tol) */
    int iel_no_shadow;  /* 0scf: 0 the energy and forces of the shadow potential U(R, x + delta) -
                           U_es(0, delta) (the reference's default, exact and conserved); 1 the
                           fixed-dipole energy and forces at mu */
    /* The local preconditioner of the CG (Induction.local_cut / local_niter, forcefield.py:302-305,
       1766-1792): z = M^-1 r by local_niter inner CG iterations on alpha^-1 v + the row field of v
       over the entries closer than local_cut (at most 48 per atom: PGM_STATUS_SHORT_OVERFLOW),
       started from alpha r; the outer CG is then flexible.  local_niter 0: Jacobi (the default).
       Not with iel. */
    double local_cut;   /* [nm], below the (electrostatics) cutoff */
    int local_niter;    /* 0..8 */
} PgmSettings;

/* One system of the batch: topology and parameters (host arrays, copied at creation). */
typedef struct {
    int n_atoms;
    int n_mol;
    const int32_t *mol_start;   /* (n_mol + 1) first atom of every molecule; molecules contiguous */
    const double *q;            /* (n_atoms) [e] */
    const double *radius;       /* (n_atoms) Gaussian radii [nm] */
    const double *alpha;        /* (n_atoms) polarizabilities [nm^3], > 0 */
    const double *lj_rmin_half; /* (n_atoms) LJ R* [nm] */
    const double *lj_sqrt_eps;  /* (n_atoms) [sqrt(kJ/mol)] */
    const double *masses;       /* (n_atoms) [amu] (molecular virial) */
    int n_cov;
    const int32_t *cov_i;       /* (n_cov) atom carrying the covalent dipole (local index) */
    const int32_t *cov_j;       /* (n_cov) atom it points to (local index) */
    const double *cov_c;        /* (n_cov) strength [e nm] */
    int pme_grid[3];            /* K1, K2, K3: even, factors 2, 3, 5 only, <= 256 */
    double box0[9];             /* a box of the run, to size the cell grid [nm] */
} PgmSystemDesc;

/* Induced-dipole solver state (InductionState, forcefield.py:679-713), device pointers, in/out. */
typedef struct {
    double *mu;      /* (N, 3) converged dipoles of the last solve [e nm] */
    double *hist;    /* (4, N, 3) dipoles of the last steps, newest first */
    int32_t *count;  /* (n_systems) steps recorded */
    double *norm;    /* (n_systems) mean|alpha b| of the last unfused step */
    double *xl;      /* iel only: (pgm_iel_len(order), N, 3) auxiliary dipoles, newest first
                        (InductionState.xl); NULL otherwise */
} PgmInduction;

/* Outputs of a step (Result, forcefield.py:716-746), device pointers; any may be NULL. */
typedef struct {
    double *energy;       /* (n_systems, 3) elec, vdw, total [kJ/mol] */
    double *forces;       /* (N, 3) [kJ/mol/nm] */
    double *virial;       /* (n_systems, 3, 3) dE/d eps at fixed mu minus the LJ tail impulse [kJ/mol] */
    int32_t *iterations;  /* (n_systems) CG iterations */
    double *residual;     /* (n_systems) max|alpha r| / norm before the peek step */
    uint32_t *status;     /* (n_systems) PGM_STATUS_* bits */
} PgmOutputs;

typedef struct PgmHandle PgmHandle;

/* Auxiliary dipoles kept by an iEL state of this order: x_{n+1} and x_n ... x_{n-K}, at least 3
 * (PGMForceField.xl_len, forcefield.py:1476-1479). */
int pgm_iel_len(int order);

/* PGMForceField.__init__ (forcefield.py:868): settings and the systems of the batch. */
PgmStatus pgm_create(const PgmSettings *settings, const PgmSystemDesc *systems, int n_systems, int device,
                     PgmHandle **out);
PgmStatus pgm_destroy(PgmHandle *h);

/* PGMForceField.compute (forcefield.py:2489): solve the induced dipoles from the predictor state,
 * then energies, forces and the molecular virial (strain_derivative, forcefield.py:2628, at the
 * returned mu).  pos (N, 3), box (n_systems, 3, 3).  idx: candidate partners (N, idx_width),
 * padding N_system (the reference's neighbour-list rows, local indices), or NULL to let the engine
 * find the pairs with its own cell list.  stream: a cudaStream_t (NULL: the legacy stream). */
PgmStatus pgm_compute(PgmHandle *h, void *stream, const double *pos, const double *box, const int32_t *idx,
                      int idx_width, PgmInduction *ind, PgmOutputs *out);

/* pgm_compute with host pointers (copies in and out; ind arrays and out arrays on the host).
 * ind == NULL keeps the induction state on the device, in the handle: each call starts from the
 * state the previous pgm_compute_host call left (empty before the first: no history, count 0), and
 * only positions, box and the outputs cross the host link -- the layout of a host MD engine that
 * owns the coordinates but not the solver's state (the reference keeps InductionState in device
 * arrays).  A call with ind set loads that state and leaves it (updated) in the handle too. */
PgmStatus pgm_compute_host(PgmHandle *h, const double *pos, const double *box, PgmInduction *ind, PgmOutputs *out);

/* PGMForceField.energy (forcefield.py:2562): energy only, CG started from ind->mu (plain start), no
 * history push; ind->mu receives the converged dipoles.  energy (n_systems, 3). */
PgmStatus pgm_energy(PgmHandle *h, void *stream, const double *pos, const double *box, const int32_t *idx,
                     int idx_width, PgmInduction *ind, double *energy, int32_t *iterations, uint32_t *status);

/* PGMForceField.energy_fixed_mu + strain_derivative (forcefield.py:2249, 2628): energies (n_systems,
 * 3), forces (N, 3) and molecular virial (n_systems, 3, 3) with the induced dipoles held at mu
 * (N, 3).  Any output may be NULL. */
PgmStatus pgm_energy_fixed_mu(PgmHandle *h, void *stream, const double *pos, const double *box, const int32_t *idx,
                              int idx_width, const double *mu, double *energy, double *forces, double *virial,
                              uint32_t *status);

/* PGMForceField._field (forcefield.py:1428): the total field -dU/dd (N, 3) [e/nm^2] of charges
 * (q != 0: the system's charges; 0: none) and dipoles d (N, 3). */
PgmStatus pgm_field(PgmHandle *h, void *stream, const double *pos, const double *box, int with_charges,
                    const double *d, double *field);

/* PGMForceField.size_rows / grow_rows (forcefield.py:1269-1296): set the row capacity (pairs per
 * row, rounded up to a multiple of 32); 0 restores the automatic size. */
PgmStatus pgm_set_row_capacity(PgmHandle *h, int capacity);
int pgm_row_capacity(const PgmHandle *h);

/* Candidates kept per atom in the engine's Verlet list (rounded up to a multiple of 32; 0:
 * automatic); the list is rebuilt at the next call. */
/* Split rows: the electrostatic part of the row capacity (PGM_ERR_INVALID without split rows) and
 * the largest van der Waals part of the last row build. */
PgmStatus pgm_set_elec_capacity(PgmHandle *h, int capacity);
int pgm_elec_capacity(const PgmHandle *h);
int pgm_max_vdw_count(PgmHandle *h);
PgmStatus pgm_set_list_capacity(PgmHandle *h, int capacity);
int pgm_list_capacity(const PgmHandle *h);
/* Steps since creation at which the candidate list was rebuilt (host counter of calls that found
 * the rebuild flag set is not kept; this reads the device counter). */
long long pgm_list_rebuilds(PgmHandle *h);

/* Largest in-cutoff pair count of any row in the last step (for size_rows). */
int pgm_max_row_count(PgmHandle *h);

/* Total atoms, systems. */
int pgm_num_atoms(const PgmHandle *h);
int pgm_num_systems(const PgmHandle *h);

/* Text of the last error of this thread. */
const char *pgm_last_error(void);

/* Kernels launched by the last pgm_compute / pgm_energy / pgm_field call, counting one CG iteration
 * when the call was captured into a CUDA graph (the loop then runs as a conditional while node),
 * and the kernels of one CG iteration (launch accounting). */
long long pgm_last_launch_count(const PgmHandle *h);
long long pgm_launches_per_iteration(const PgmHandle *h);
/* CG iterations of a captured solve that run as plain graph nodes ahead of its conditional while
 * node (from the iteration count of the last host-driven solve; 0: all in the while node). */
int pgm_unrolled_iterations(const PgmHandle *h);

/* Average duration [ms] of one launch of a kernel of the last pgm_compute, re-run `reps` times on
 * `stream` between CUDA events on the state that step left: 0 the CG matvec (row field + PME
 * gather in one kernel), 1 the PME spread, 2 the five FFT/convolution passes, 3 the energy/force
 * pass, 4 the row build, 5 the first FFT pass alone, 6 a spread followed by the first FFT pass,
 * 7 the row field alone, 8 the PME gather + operator assembly alone, 9 a whole operator sweep as
 * the solver runs it (spread, row field beside the FFT chain, gather), 10 the learned guess's
 * channel pass, 11 its feature pass, 12 its model.  The last pgm_compute's position (and, for 10,
 * induction history) arrays must still be valid. */
PgmStatus pgm_profile_kernel(PgmHandle *h, void *stream, int which, int reps, double *ms_per_launch);

/* In-cutoff pairs (both rows of every pair) of the last step's row build. */
long long pgm_row_pairs(PgmHandle *h);

/* ------------------------------------------------------------------ learned initial guess
 * No counterpart in the reference (its guesses are the mu3 / mu4 / ls predictors,
 * forcefield.py:1917-2008).  A message-passing model on the short-range graph (edges r < the graph
 * cutoff) predicts the correction mu* - x4 to the mu4 extrapolation x4 of the converged dipoles,
 * from the change of the graph's permanent field since the last step and the last steps' dipoles.
 * With predictor 5 the solve starts from x4 + the prediction, with mu4's fused start (one field
 * sweep), and CG iterates to the same tolerance; the untrained (zero) model is mu4.
 * Per-atom channels (N, 12) floats: c0 = alpha (b - b_prev) (b: the real-space field of charges and
 * permanent dipoles over the graph), c1 = mu1 - mu2, c2 = x4 - mu1, mu1.  Features: 16 rotation
 * invariants (float, (N, 16)) and 15 vector channels (float, (N, 15, 3)): c0..c2 and their
 * radial-basis sums over the graph, plain and projected on the edge direction.  The model
 * (pgm_nn_param_count() floats, device) is the MLP of pgm_nn_predict; sigma is the scale of the
 * per-step changes in the invariants [e nm]. */
PgmStatus pgm_set_nn_model(PgmHandle *h, const float *weights, float sigma, float graph_cutoff);
/* ------------------------------------------------------------------ autotuner
 * No counterpart in the reference (XLA chooses its own fusions).  The kernel variants of a handle:
 * rowfield_lanes, the lanes that share one neighbour row in the CG matvec's row stream (32: a warp
 * per atom; 16, 8: two or four atoms per warp); forces_blocks_per_sm, the force pass's register
 * budget, as resident blocks of 256 threads per SM (2, 3, 4: registers against warps); sweep_early, the
 * order of the CG sweep's concurrent parts; rowfield_grid, the row field beside the FFT chain on
 * every SM (0) or on 4 or 8 blocks per SM (1, 2) at the highest priority, the FFT passes filling the rest
 * of each SM.  Unless fixed by
 * pgm_set_tuning, the first pgm_compute that is not being captured times every variant on its own
 * rows (CUDA events on its stream, the mean of 10 launches after one) and keeps the fastest;
 * handles of the same precision, order, atoms, row capacity and grid size in one process share the
 * result (from_cache).  Every variant computes the same sums (in another order of addition). */
typedef struct {
    int rowfield_lanes;        /* 32, 16 or 8 (default 32 before tuning) */
    int forces_blocks_per_sm;  /* 2, 3 or 4 (default 3) */
    double rowfield_ms[3];     /* timed launches: 32, 16, 8 lanes [ms] */
    double forces_ms[3];       /* timed launches: 2, 3, 4 blocks per SM [ms] */
    int tuned;                 /* 1 once timed (or taken from the cache) */
    int from_cache;
    int sweep_early;           /* the CG direction's sweep: 0 the row field forked after the spread
                                  (on p), 1 at the start of the sweep (on z; the rows of p = z +
                                  beta p_prev combined in the gather) */
    double sweep_ms[2];        /* timed sweeps of the two schedules [ms] */
    int rowfield_grid;         /* 0 (one block per 8 rows), 1 or 2: 4 or 8 blocks per SM beside the FFT chain */
    double grid_ms[3];         /* timed sweeps with rowfield_grid 0, 1, 2 [ms] */
} PgmTuning;
PgmStatus pgm_tuning(PgmHandle *h, PgmTuning *out);
/* Fix the variants (0, or -1 for sweep_early and rowfield_grid, leaves one as it is; all so:
 * autotune again at the next direct step). */
PgmStatus pgm_set_tuning(PgmHandle *h, int rowfield_lanes, int forces_blocks_per_sm, int sweep_early, int rowfield_grid);
/* Time the variants now on the last step's rows (synchronises the stream). */
PgmStatus pgm_autotune(PgmHandle *h, void *stream);

/* The learned guess's fallback (no counterpart in the reference, whose solver has no learned
 * guess): with predictor 5 every solve starts from x4 + the model's correction with the fused start,
 * whose residual r0 is known before the first CG iteration at no extra cost.  When max|alpha r0| /
 * norm exceeds `factor` times the running mean of the same quantity for starts from the plain
 * extrapolation x4 (recorded from the solves without the model and from every fallback), that
 * system restarts from x4: r0 += A delta, one operator sweep of the correction delta (captured in a
 * conditional node that runs only then).  factor 0 turns the check off; default 2. */
PgmStatus pgm_set_nn_fallback(PgmHandle *h, double factor);
/* Per system (host arrays of n_systems, either may be NULL): the number of fallbacks so far and the
 * recorded mean start residual of the extrapolation (-1 before the first record). */
PgmStatus pgm_nn_fallback_stats(PgmHandle *h, long long *fallbacks, double *ref_err);
/* Features at a geometry: hist (4, N, 3) device (newest first, as PgmInduction.hist); bl_prev (N, 4)
 * floats, the graph's permanent field of the previous step, or NULL (c0 = 0); bl_out (N, 4)
 * receives this step's; inv, vec device.  Uses the sigma and graph cutoff of pgm_set_nn_model
 * (before any: 2e-4 e nm and 0.5 nm). */
PgmStatus pgm_nn_features(PgmHandle *h, void *stream, const double *pos, const double *box, const double *hist,
                          const float *bl_prev, float *bl_out, float *inv, float *vec);
int pgm_nn_param_count(void);
/* mu (n, 3) = sum_c c_c(inv) vec_c with c = MLP(inv): BF16 tensor cores, FP32 accumulation. */
PgmStatus pgm_nn_predict(void *stream, const float *weights, const float *inv, const float *vec, int n, float *mu);
/* Training: loss += sum |mu - target|^2 * inv_scale (double, device) and grad += dloss/dweights. */
PgmStatus pgm_nn_loss_grad(void *stream, const float *weights, const float *inv, const float *vec, const float *target, int n,
                           float inv_scale, float *grad, double *loss);
/* One Adam step (bias-corrected at `step` >= 1) on the weights; clears grad. */
PgmStatus pgm_nn_adam(void *stream, float *weights, float *grad, float *m, float *v, float lr, float beta1, float beta2,
                      float eps, int step);
const char *pgm_nn_last_error(void);

/* ------------------------------------------------------------------ message-passing guess
 * No counterpart in the reference.  The 2-layer message-passing model of the learned guess on the
 * graph of the row entries closer than graph_cutoff (pgm_mpnn.cu): h0 = SiLU(W0 inv + b0) (16 ->
 * 64); per layer a continuous-filter convolution: g = W_g h (16 features), a_i[f] = sum_r
 * W_f[f, r] sum over the graph of phi_r(d_ij) g_j[f] (phi_r: 8 Gaussians times a cosine cutoff),
 * h += W_b SiLU(W_a [h; a] + b_a) + b_b (80 -> 64 -> 64); c = W_o h + b_o (16); mu = sigma sum_c
 * c_c v_c over the 15 vector channels.  BF16 weights and activations, FP32 accumulation on the
 * tcgen05 tensor cores.  Weights: pgm_mpnn_param_count() FP32 (W0, b0, then per layer Wg, Wf, Wa,
 * ba, Wb, bb, then Wo, bo; matrices out x in, row-major). */
int pgm_mpnn_param_count(void);
/* Use it as the learned guess of predictor 5 (weights device FP32; NULL: no model). */
PgmStatus pgm_set_mpnn_model(PgmHandle *h, const float *weights, float sigma, float graph_cutoff);
/* The graph of the last step with predictor 5: edges (N, emax) float4 (x_i - x_j, y, z, partner j
 * as the bits of an int32) and counts (N) (a count above emax: the first emax kept). */
PgmStatus pgm_nn_graph(PgmHandle *h, void *stream, void *edges, int *counts, int emax);
/* Device workspace of pgm_mpnn_predict (train 0) or pgm_mpnn_loss_grad (train 1) for n atoms [bytes]. */
long long pgm_mpnn_work_bytes(int n, int train);
/* Prediction mu (n, 3) from invariants inv (n, 16), channels vec (n, 15, 3) and a symmetric graph
 * (edges (n, emax), counts (n) as pgm_nn_graph writes). */
PgmStatus pgm_mpnn_predict(void *stream, const float *weights, const float *inv, const float *vec, const void *edges,
                           const int *ecount, int emax, int n, float sigma, float graph_cutoff, void *work, float *mu);
/* Training: loss += scale sum |mu - target|^2 (double, device) and grad += dloss/dweights (FP32,
 * device), the forward and activation gradients on the tensor cores, the weight gradients as FP32
 * sums over the atoms. */
PgmStatus pgm_mpnn_loss_grad(void *stream, const float *weights, const float *inv, const float *vec, const float *target,
                             const void *edges, const int *ecount, int emax, int n, float sigma, float graph_cutoff,
                             float scale, void *work, float *grad, double *loss);
/* One Adam step (bias-corrected at `step` >= 1) on the message-passing model's weights; clears grad. */
PgmStatus pgm_mpnn_adam(void *stream, float *weights, float *grad, float *m, float *v, float lr, float beta1, float beta2,
                        float eps, int step);
const char *pgm_mpnn_last_error(void);

/* ------------------------------------------------------------------ tcgen05 dense layers
 * No counterpart in the reference (its learned models run through XLA).  C = act(A W^T + bias) on
 * the 5th-generation tensor cores: A (M, lda) BF16 with the first K of every row used (lda a
 * multiple of 8), W (N, K) BF16, bias N floats or NULL, C (M, ldc) FP32 (out_f32, ldc a multiple of
 * 4) or BF16 (ldc a multiple of 8); A, W and C 16-byte aligned, else PGM_ERR_INVALID; act 0
 * none, 1 SiLU; BF16 products accumulated in FP32 (tensor memory).  Compiled (K, N): (16, 64),
 * (64, 64), (64, 128), (80, 64), (64, 32), (128, 16); others return PGM_ERR_UNSUPPORTED.  *err
 * (device int) is set when a tile's wait for its MMAs gave up (it is never expected to). */
PgmStatus pgm_tc_gemm(void *stream, int K, int N, int act, int out_f32, const void *A, int lda, int M, const void *W,
                      const float *bias, void *C, int ldc, int *err);
const char *pgm_tc_last_error(void);

/* ------------------------------------------------------------------ allocation-free field
 * pgm_field_static has no counterpart in the reference.  It is for callers that must not allocate
 * device memory: a jax.ffi custom call inside XLA (XLA has reserved most of the GPU memory for its
 * own allocator and passes the call all the buffers it may use) or code recording a CUDA graph.  It
 * computes the same total field -dU/dd (N, 3) [e/nm^2] as pgm_field, in FP64, for one system, with
 * every intermediate in one static device array of the library (1 MB, held by each GPU that loads
 * the library until exit) and no handle: no cudaMalloc, cudaFree or allocating library call.
 * All pointers are device pointers: pos (N, 3), box (3, 3), q and radius (N), d (N, 3), field (N, 3).
 * Limits: N <= PGM_STATIC_MAX_ATOMS, each mesh size <= PGM_STATIC_MAX_K with K1 K2 K3 <=
 * PGM_STATIC_MAX_GRID, order 4, 6 or 8; larger inputs return PGM_ERR_UNSUPPORTED with a message in
 * pgm_static_last_error().  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and should come before any stream capture.  All calls share the array:
 * calls that overlap on the GPU (other streams or threads at the same time) race on it.
 * The stream must belong to the current device (PGM_ERR_INVALID otherwise); a CUDA error left
 * pending by an earlier launch is reported (PGM_ERR_CUDA) and not cleared.  The box must be lower
 * triangular with a positive diagonal and the cutoff at most half its smallest diagonal element:
 * the box is on the device, so this is checked there and any other box gives a NaN field.  Pairs
 * are taken by minimum image within the cutoff; pgm_field's rows also keep the pairs of one
 * molecule beyond the cutoff, so the two differ for a molecule larger than the cutoff. */
#define PGM_STATIC_MAX_ATOMS 4096
#define PGM_STATIC_MAX_K 64
#define PGM_STATIC_MAX_GRID 32768
PgmStatus pgm_field_static(void *stream, int n_atoms, const double *pos, const double *box, const double *q,
                           const double *radius, double cutoff, double ewald_beta, const int *pme_grid, int pme_order,
                           int with_charges, const double *d, double *field);
const char *pgm_static_last_error(void);

/* ------------------------------------------------------------------ rigid-molecule MD driver
 * The caller of the force field in the MD benchmarks: the rigid-body step of pgm_jax/md/
 * integrate.py:743-761 (B A O A B) with md/rigid.py bodies and the Langevin O-step of
 * md/thermostats.py:195-240.  Bodies: centre of mass X (M, 3), quaternion q (M, 4, body -> space,
 * w first), momentum P (M, 3) and body-frame angular momentum L (M, 3), device arrays; atoms at
 * X + R(q) b_i with `body` b (N, 3) in each molecule's principal frame and `inertia` (M, 3) its
 * principal moments.  Units amu, nm, ps, kJ/mol. */
typedef struct PgmRigid PgmRigid;

PgmStatus pgm_rigid_create(int n_mol, const int32_t *mol_start, const int32_t *mol_system, const double *masses,
                           const double *body, const double *inertia, int device, PgmRigid **out);
PgmStatus pgm_rigid_destroy(PgmRigid *r);

/* Kick (with the forces of the previous step; NULL: none), then with gamma [1/ps] > 0: half drift,
 * Langevin (kT [kJ/mol] per system, device; the noise is drawn from (seed, the handle's step
 * counter)), half drift; with gamma = 0 (NVE): one drift of dt (the reference's velocity Verlet,
 * integrate.py:743-761).  A drift moves the centres and turns the bodies by the free-rotor splitting
 * (axes 3, 2, 1, 2, 3).  Writes the atom positions pos (N, 3) for the next force call.  box
 * (n_systems, 3, 3) keeps the centres in the box. */
PgmStatus pgm_rigid_begin_step(PgmRigid *r, void *stream, double dt, double gamma, const double *kT, uint64_t seed,
                               const double *forces, double *com, double *quat, double *mom, double *angmom, double *pos,
                               const double *box);
/* Set the step counter of the Langevin noise (it advances by one at every pgm_rigid_end_step). */
PgmStatus pgm_rigid_set_step(PgmRigid *r, uint64_t step);
/* Closing half kick with the new forces. */
PgmStatus pgm_rigid_end_step(PgmRigid *r, void *stream, double dt, const double *forces, const double *quat, double *mom,
                             double *angmom);
/* Kinetic energy per system (device, n_systems). */
PgmStatus pgm_rigid_kinetic(PgmRigid *r, void *stream, const double *mom, const double *angmom, double *ke);
/* Momenta and angular momenta of each system's molecules times factor[system] (device,
 * n_systems): the sqrt(T_new / T_old) rescaling of a replica exchange (pgm_jax/md/remd.py:571-611). */
PgmStatus pgm_rigid_scale_momenta(PgmRigid *r, void *stream, const double *factor, double *mom, double *angmom);
const char *pgm_rigid_last_error(void);

/* ------------------------------------------------------------------ path-integral MD
 * The ring-polymer integrator around the batched force field (pgm_jax/md/pimd.py:484-700): the P
 * beads are the systems of one engine batch, positions / momenta / forces bead-major (atom i of
 * bead k at k N + i, (P N, 3) doubles).  A step: pgm_pimd_kick(dt/2), pgm_pimd_free_thermostat
 * (Cayley A(dt/2), PILE-L O(dt), A(dt/2) in normal modes), the force call on all beads (+
 * pgm_water_bonded for flexible water), pgm_pimd_kick(dt/2). */
/* mom += h forces over n3 = 3 P N doubles. */
PgmStatus pgm_pimd_kick(void *stream, long long n3, double h, const double *forces, double *mom);
/* A O A in normal modes (pimd.py:222-296, 411-440): C (P, P) row-major normal-mode matrix
 * (C[j][l], bead j, mode l), omega (P,) mode frequencies [rad/ps], gamma (P,) frictions [1/ps]
 * (all 0: RPMD), mass (N,) [amu], kT_P = P kB T [kJ/mol]; the noise is drawn from (seed, *counter),
 * and the device counter advances by one.  1 <= P <= 32.  All pointers device. */
PgmStatus pgm_pimd_free_thermostat(void *stream, int beads, int n_atoms, const double *C, const double *omega, const double *gamma,
                                   const double *mass, double dt, double kT_P, uint64_t seed, uint64_t *counter, double *pos,
                                   double *mom);
/* PILE-G (pimd.py:411-440 with the Bussi step of thermostats.py:279-335): the rescaling factor of
 * the ring polymer's centroid for an O step of length dt [ps] with time constant tau [ps], from the
 * centroid kinetic energy of mom at kT_P with N_f = 3 n_atoms degrees of freedom; random numbers
 * from (seed, *counter) (the counter is not advanced).  work: 4 device doubles, written as
 * [K, alpha, R1, S] (the kinetic energy, the factor, the normal and the chi^2(N_f - 1) draws). */
PgmStatus pgm_pimd_centroid_bussi(void *stream, int beads, int n_atoms, const double *C, const double *mass, double dt, double kT_P,
                                  double tau, uint64_t seed, const uint64_t *counter, const double *mom, double *work);
/* pgm_pimd_free_thermostat with the centroid mode multiplied by *centroid_scale (device; the
 * factor pgm_pimd_centroid_bussi left in work[1]) in place of its Langevin step (its friction
 * should be 0); centroid_scale NULL: pgm_pimd_free_thermostat. */
PgmStatus pgm_pimd_free_thermostat_scaled(void *stream, int beads, int n_atoms, const double *C, const double *omega,
                                          const double *gamma, const double *mass, double dt, double kT_P, uint64_t seed,
                                          uint64_t *counter, double *pos, double *mom, const double *centroid_scale);
/* q-TIP4P/F intramolecular water term (pgm_jax/models/water.py:33-69) for molecules O, H, H at
 * first_atom[m]: params (host, 5) = D [kJ/mol], alpha [1/nm], r_eq [nm], k_theta [kJ/mol/rad^2],
 * theta_eq [rad]; forces += its forces; energy[mol_system[m]] += its energy (energy may be NULL). */
PgmStatus pgm_water_bonded(void *stream, int n_mol, const int32_t *first_atom, const int32_t *mol_system, const double *pos,
                           const double *params, double *forces, double *energy);
const char *pgm_pimd_last_error(void);

/* Stream capture of engine calls into a replayable CUDA graph (exec is a cudaGraphExec_t). */
PgmStatus pgm_graph_begin(void *stream);
PgmStatus pgm_graph_end(void *stream, void **exec_out);
PgmStatus pgm_graph_launch(void *exec, void *stream);
PgmStatus pgm_graph_destroy(void *exec);

#ifdef __cplusplus
}
#endif
#endif
