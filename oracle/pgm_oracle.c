/*
 * pgm_oracle.c -- TEST INFRASTRUCTURE, NOT THE PRODUCT (see pgm_oracle.h).
 *
 * A plain FP64 restatement, with OpenMP over atoms, of the per-step pGM electrostatics of
 * pGM-JAX.  Every function names the reference code it follows.  The structure is deliberately
 * plain (a cell-list pair search with the reference's minimum image, a recursive mixed-radix FFT,
 * OpenMP over atoms, grid slabs and FFT lines): it is a checker and a CPU baseline.
 */
#include "pgm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KE 138.935458 /* kJ mol^-1 nm e^-2, pgm_jax/units.py:31 */

static int set_threads(const pgmo_settings *s);
#define SQRT_PI 1.7724538509055160273

/* ------------------------------------------------------------------ box helpers (md/box.py) */
/* Sequential minimum image for a reduced lower-triangular box (box.py:130-153, and the row
 * displacements of forcefield.py:1045-1056): along c by z, then b by y, then a by x. */
static void min_image(double x[3], const double H[9]) {
    for (int c = 2; c >= 0; --c) {
        double n = nearbyint(x[c] / H[c * 3 + c]);
        for (int j = 0; j <= c; ++j) x[j] -= n * H[c * 3 + j];
    }
}

static double det3(const double H[9]) {
    return H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
           H[2] * (H[3] * H[7] - H[4] * H[6]);
}

/* Cofactor inverse (box.py:195-234). */
static void inv3(const double H[9], double Hi[9]) {
    double d = det3(H);
    Hi[0] = (H[4] * H[8] - H[5] * H[7]) / d;
    Hi[1] = (H[2] * H[7] - H[1] * H[8]) / d;
    Hi[2] = (H[1] * H[5] - H[2] * H[4]) / d;
    Hi[3] = (H[5] * H[6] - H[3] * H[8]) / d;
    Hi[4] = (H[0] * H[8] - H[2] * H[6]) / d;
    Hi[5] = (H[2] * H[3] - H[0] * H[5]) / d;
    Hi[6] = (H[3] * H[7] - H[4] * H[6]) / d;
    Hi[7] = (H[1] * H[6] - H[0] * H[7]) / d;
    Hi[8] = (H[0] * H[4] - H[1] * H[3]) / d;
}

/* ------------------------------------------------------------------ radial kernels */
/* B_n of erf(a r)/r, n = 0..3 (md/kernels.py:76-118): Taylor series (15 terms) where (a r)^2 < 1,
 * the closed-form recursion elsewhere. */
void pgmo_erf_kernels(double a, double r, double B[4]) {
    double x = a * r, s = x * x;
    double c0 = 2.0 * a / SQRT_PI, a2 = a * a;
    if (s < 1.0) {
        double t[15];
        t[0] = 1.0;
        for (int m = 1; m < 15; ++m) t[m] = t[m - 1] * (-s) / m;
        double f = 1.0;
        for (int n = 0; n < 4; ++n) {
            double acc = 0.0;
            for (int m = 0; m < 15; ++m) acc += t[m] / (2 * m + 2 * n + 1);
            B[n] = c0 * f * acc;
            f *= 2.0 * a2;
        }
    } else {
        double r2 = r * r;
        double c = c0 * exp(-s);
        B[0] = erf(x) / r;
        double f = 1.0;
        for (int n = 1; n < 4; ++n) {
            B[n] = ((2 * n - 1) * B[n - 1] - f * c) / r2;
            f *= 2.0 * a2;
        }
    }
}

/* G_n = B_n[erf(a r)/r] - B_n[erf(beta r)/r] (forcefield.py:1318-1338). */
static void pair_kernels(double a, double beta, double r, double G[4]) {
    double A[4], B[4];
    pgmo_erf_kernels(a, r, A);
    pgmo_erf_kernels(beta, r, B);
    for (int n = 0; n < 4; ++n) G[n] = A[n] - B[n];
}

/* ------------------------------------------------------------------ B-splines (md/pme.py:57-131) */
/* Orders 2..order of M_n(f + n - 1 - k) by the recursion of pme.py:81-103; theta from the last
 * order, dtheta (d/df) from order-1, d2theta from order-2. */
void pgmo_bspline(double f, int order, double *theta, double *dtheta, double *d2theta) {
    double data[32] = {0}, prev[32] = {0}, prev2[32] = {0};
    data[0] = 1.0 - f;
    data[1] = f;
    for (int n = 3; n <= order; ++n) {
        memcpy(prev2, prev, sizeof(prev));
        memcpy(prev, data, sizeof(data));
        double div = 1.0 / (n - 1.0);
        data[n - 1] = div * f * data[n - 2];
        for (int k = 1; k < n - 1; ++k)
            data[n - k - 1] = div * ((f + k) * data[n - k - 2] + (n - k - f) * data[n - k - 1]);
        data[0] = div * (1.0 - f) * data[0];
    }
    /* prev = order-1 values (length order-1), prev2 = order-2 values */
    for (int k = 0; k < order; ++k) {
        theta[k] = data[k];
        double a = k >= 1 ? prev[k - 1] : 0.0, b = k < order - 1 ? prev[k] : 0.0;
        dtheta[k] = a - b;
        double c0 = k >= 2 ? prev2[k - 2] : 0.0, c1 = (k >= 1 && k - 1 < order - 2) ? prev2[k - 1] : 0.0,
               c2 = k < order - 2 ? prev2[k] : 0.0;
        if (d2theta) d2theta[k] = c0 - 2.0 * c1 + c2;
    }
}

/* |sum_j M_p(j+1) exp(2 pi i m j / K)|^2 with OpenMM's patch of near-zero values (pme.py:106-131). */
static void bspline_moduli(int K, int order, double *mod) {
    double th[32], dth[32];
    pgmo_bspline(0.0, order, th, dth, NULL);
    for (int m = 0; m < K; ++m) {
        double c = 0.0, s = 0.0;
        for (int j = 0; j < order; ++j) {
            double arg = 2.0 * M_PI * m * j / K;
            c += th[j] * cos(arg);
            s += th[j] * sin(arg);
        }
        mod[m] = c * c + s * s;
    }
    for (int m = 0; m < K; ++m)
        if (mod[m] < 1e-7) mod[m] = 0.5 * (mod[(m - 1 + K) % K] + mod[(m + 1) % K]);
}

/* ------------------------------------------------------------------ FFT (recursive mixed radix) */
/* w[j] = exp(sign 2 pi i j / L), j < L: the twiddles of every sub-transform of a length-L line. */
static double complex *twiddles(int L, int sign) {
    double complex *w = malloc(sizeof(double complex) * L);
    for (int j = 0; j < L; ++j) {
        double ang = sign * 2.0 * M_PI * (double)j / L;
        w[j] = cos(ang) + I * sin(ang);
    }
    return w;
}

/* Decimation in time by the smallest prime factor p of n: p sub-transforms of length n / p of the
 * strided input, then the p-point butterflies.  w is the twiddle table of the full line length
 * (wstep = L / n), work holds 2 n values (this level's sub-transforms and the levels below). */
static void fft_rec(const double complex *x, int n, int stride, double complex *out, const double complex *w, int wstep,
                    double complex *work) {
    if (n == 1) {
        out[0] = x[0];
        return;
    }
    int p = 2;
    while (p * p <= n && n % p) ++p;
    if (n % p) p = n; /* prime */
    int m = n / p;
    double complex *sub = work;
    for (int r = 0; r < p; ++r) fft_rec(x + r * stride, m, stride * p, sub + r * m, w, wstep * p, work + n);
    for (int k = 0; k < m; ++k)
        for (int s2 = 0; s2 < p; ++s2) {
            int kk = k + m * s2;
            double complex acc = 0;
            for (int r = 0; r < p; ++r) acc += sub[r * m + k] * w[(size_t)((long long)r * kk % n) * wstep];
            out[kk] = acc;
        }
}

/* In-place unnormalised 3D DFT, sign -1 forward, +1 backward, grid [K0][K1][K2]. */
static void fft3d(double complex *g, const int K[3], int sign, int nth) {
    int K0 = K[0], K1 = K[1], K2 = K[2];
    (void)nth;
    double complex *w0 = twiddles(K0, sign), *w1 = twiddles(K1, sign), *w2 = twiddles(K2, sign);
#pragma omp parallel
    {
        int L = K0 > K1 ? (K0 > K2 ? K0 : K2) : (K1 > K2 ? K1 : K2);
        double complex *in = malloc(sizeof(double complex) * L), *out = malloc(sizeof(double complex) * L);
        double complex *work = malloc(sizeof(double complex) * 2 * L);
#pragma omp for collapse(2)
        for (int a = 0; a < K0; ++a)
            for (int b = 0; b < K1; ++b) {
                double complex *line = g + ((size_t)a * K1 + b) * K2;
                memcpy(in, line, sizeof(double complex) * K2);
                fft_rec(in, K2, 1, out, w2, 1, work);
                memcpy(line, out, sizeof(double complex) * K2);
            }
#pragma omp for collapse(2)
        for (int a = 0; a < K0; ++a)
            for (int c = 0; c < K2; ++c) {
                for (int b = 0; b < K1; ++b) in[b] = g[((size_t)a * K1 + b) * K2 + c];
                fft_rec(in, K1, 1, out, w1, 1, work);
                for (int b = 0; b < K1; ++b) g[((size_t)a * K1 + b) * K2 + c] = out[b];
            }
#pragma omp for collapse(2)
        for (int b = 0; b < K1; ++b)
            for (int c = 0; c < K2; ++c) {
                for (int a = 0; a < K0; ++a) in[a] = g[((size_t)a * K1 + b) * K2 + c];
                fft_rec(in, K0, 1, out, w0, 1, work);
                for (int a = 0; a < K0; ++a) g[((size_t)a * K1 + b) * K2 + c] = out[a];
            }
        free(in);
        free(out);
        free(work);
    }
    free(w0);
    free(w1);
    free(w2);
}

/* ------------------------------------------------------------------ PME (md/pme.py:175-411) */
typedef struct {
    int K[3], p;
    double beta, Hinv[9], escale[9], vol;
    double *G;           /* influence on the full spectrum (K0 K1 K2), 0 at m = 0 */
    double complex *grid;
    int *base;           /* (n, 3) floor(w) */
    double *th, *dth, *d2th; /* (n, 3, p) */
} pme_t;

/* pme.py:209-241 and influence 243-267 (full spectrum instead of the rfft half; same sum). */
static void pme_init(pme_t *P, const pgmo_settings *s, const double *H, int n) {
    memcpy(P->K, s->K, sizeof(P->K));
    P->p = s->order;
    P->beta = s->beta;
    inv3(H, P->Hinv);
    P->vol = fabs(det3(H));
    for (int b = 0; b < 3; ++b)
        for (int a = 0; a < 3; ++a) P->escale[b * 3 + a] = P->Hinv[b * 3 + a] * P->K[a];
    int K0 = P->K[0], K1 = P->K[1], K2 = P->K[2];
    size_t ng = (size_t)K0 * K1 * K2;
    P->G = malloc(sizeof(double) * ng);
    P->grid = malloc(sizeof(double complex) * ng);
    double *mod[3];
    for (int a = 0; a < 3; ++a) {
        mod[a] = malloc(sizeof(double) * P->K[a]);
        bspline_moduli(P->K[a], P->p, mod[a]);
    }
    /* reciprocal vectors: rows of inv(H)^T, i.e. R[a][c] = Hinv[c][a] */
    for (int i = 0; i < K0; ++i)
        for (int j = 0; j < K1; ++j)
            for (int k = 0; k < K2; ++k) {
                int m[3] = {i <= (K0 - 1) / 2 ? i : i - K0, j <= (K1 - 1) / 2 ? j : j - K1,
                            k <= (K2 - 1) / 2 ? k : k - K2};
                /* np.fft.fftfreq(K, 1/K): K/2 maps to -K/2 for even K */
                if (K0 % 2 == 0 && i == K0 / 2) m[0] = -K0 / 2;
                if (K1 % 2 == 0 && j == K1 / 2) m[1] = -K1 / 2;
                if (K2 % 2 == 0 && k == K2 / 2) m[2] = -K2 / 2;
                double mv[3];
                for (int c = 0; c < 3; ++c)
                    mv[c] = m[0] * P->Hinv[c * 3 + 0] + m[1] * P->Hinv[c * 3 + 1] + m[2] * P->Hinv[c * 3 + 2];
                double msq = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
                size_t id = ((size_t)i * K1 + j) * K2 + k;
                if (msq > 0) {
                    double g = exp(-M_PI * M_PI * msq / (P->beta * P->beta)) / (2 * M_PI * P->vol * msq);
                    P->G[id] = g / (mod[0][i] * mod[1][j] * mod[2][k]);
                } else
                    P->G[id] = 0.0;
            }
    for (int a = 0; a < 3; ++a) free(mod[a]);
    P->base = malloc(sizeof(int) * 3 * n);
    P->th = malloc(sizeof(double) * 3 * n * P->p);
    P->dth = malloc(sizeof(double) * 3 * n * P->p);
    P->d2th = malloc(sizeof(double) * 3 * n * P->p);
}

static void pme_free(pme_t *P) {
    free(P->G);
    free(P->grid);
    free(P->base);
    free(P->th);
    free(P->dth);
    free(P->d2th);
}

/* pme.py:269-304: fractional coordinates in FP64, w = K frac(u), base = floor(w), f = w - base. */
static void pme_setup(pme_t *P, const double *pos, int n) {
    int p = P->p;
#pragma omp parallel for
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            double u = pos[i * 3 + 0] * P->Hinv[0 * 3 + a] + pos[i * 3 + 1] * P->Hinv[1 * 3 + a] +
                       pos[i * 3 + 2] * P->Hinv[2 * 3 + a];
            double w = (u - floor(u)) * P->K[a];
            double b = floor(w);
            P->base[i * 3 + a] = (int)b;
            size_t o = ((size_t)i * 3 + a) * p;
            pgmo_bspline(w - b, p, P->th + o, P->dth + o, P->d2th + o);
        }
}

static inline size_t pme_index(const pme_t *P, int i, int k1, int k2, int k3) {
    int i1 = (P->base[i * 3 + 0] + k1) % P->K[0];
    int i2 = (P->base[i * 3 + 1] + k2) % P->K[1];
    int i3 = (P->base[i * 3 + 2] + k3) % P->K[2];
    return ((size_t)i1 * P->K[1] + i2) * P->K[2] + i3;
}

/* Spread q and d on the grid (pme.py:306-337).  Each thread owns a slab of k1 planes and adds, in
 * atom order, the stencil points that fall in it, so every grid value is the same ordered sum as
 * in a serial loop over the atoms.  q may be NULL. */
static void pme_spread(pme_t *P, const double *q, const double *d, int n) {
    int p = P->p;
    size_t ng = (size_t)P->K[0] * P->K[1] * P->K[2];
    memset(P->grid, 0, sizeof(double complex) * ng);
#pragma omp parallel
    {
        int nt = 1, t = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        t = omp_get_thread_num();
#endif
        int lo = (int)((long long)P->K[0] * t / nt), hi = (int)((long long)P->K[0] * (t + 1) / nt);
        for (int i = 0; i < n; ++i) {
            double e[3];
            for (int a = 0; a < 3; ++a)
                e[a] = d[i * 3 + 0] * P->escale[0 * 3 + a] + d[i * 3 + 1] * P->escale[1 * 3 + a] +
                       d[i * 3 + 2] * P->escale[2 * 3 + a];
            const double *t1 = P->th + (size_t)(i * 3 + 0) * p, *t2 = P->th + (size_t)(i * 3 + 1) * p,
                         *t3 = P->th + (size_t)(i * 3 + 2) * p;
            const double *d1 = P->dth + (size_t)(i * 3 + 0) * p, *d2 = P->dth + (size_t)(i * 3 + 1) * p,
                         *d3 = P->dth + (size_t)(i * 3 + 2) * p;
            double qi = q ? q[i] : 0.0;
            for (int a = 0; a < p; ++a) {
                int i1 = (P->base[i * 3 + 0] + a) % P->K[0];
                if (i1 < lo || i1 >= hi) continue;
                for (int b = 0; b < p; ++b)
                    for (int c = 0; c < p; ++c) {
                        double v = qi * t1[a] * t2[b] * t3[c] + e[0] * d1[a] * t2[b] * t3[c] +
                                   e[1] * t1[a] * d2[b] * t3[c] + e[2] * t1[a] * t2[b] * d3[c];
                        P->grid[pme_index(P, i, a, b, c)] += v;
                    }
            }
        }
    }
}

/* Spread q and d (pme.py:306-337), transform, return E_rec = sum G |F[Q]|^2 [e^2/nm] and leave
 * phi = dE/dQ = 2 Re IDFT(G F[Q]) (pme.py:370-376) in the real part of the grid. */
static double pme_energy_phi(pme_t *P, const double *q, const double *d, int n) {
    size_t ng = (size_t)P->K[0] * P->K[1] * P->K[2];
    pme_spread(P, q, d, n);
    fft3d(P->grid, P->K, -1, 0);
    double E = 0.0;
    for (size_t m = 0; m < ng; ++m) {
        double complex F = P->grid[m];
        E += P->G[m] * (creal(F) * creal(F) + cimag(F) * cimag(F));
        P->grid[m] = F * P->G[m];
    }
    fft3d(P->grid, P->K, +1, 0);
    for (size_t m = 0; m < ng; ++m) P->grid[m] = 2.0 * creal(P->grid[m]);
    return E;
}

/* Gradients of E_rec at atom i from phi: dU/dd (pme.py:378-388) and dU/dr (the autodiff of
 * pme.py:390-411 through the spline weights, written out with the second derivatives). */
static void pme_gather(const pme_t *P, int i, double qi, const double d[3], double gd[3], double gr[3]) {
    int p = P->p;
    double e[3];
    for (int a = 0; a < 3; ++a)
        e[a] = d[0] * P->escale[0 * 3 + a] + d[1] * P->escale[1 * 3 + a] + d[2] * P->escale[2 * 3 + a];
    const double *t1 = P->th + (size_t)(i * 3 + 0) * p, *t2 = P->th + (size_t)(i * 3 + 1) * p,
                 *t3 = P->th + (size_t)(i * 3 + 2) * p;
    const double *d1 = P->dth + (size_t)(i * 3 + 0) * p, *d2 = P->dth + (size_t)(i * 3 + 1) * p,
                 *d3 = P->dth + (size_t)(i * 3 + 2) * p;
    const double *s1 = P->d2th + (size_t)(i * 3 + 0) * p, *s2 = P->d2th + (size_t)(i * 3 + 1) * p,
                 *s3 = P->d2th + (size_t)(i * 3 + 2) * p;
    double ge[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
    for (int a = 0; a < p; ++a)
        for (int b = 0; b < p; ++b)
            for (int c = 0; c < p; ++c) {
                double ph = creal(P->grid[pme_index(P, i, a, b, c)]);
                ge[0] += ph * d1[a] * t2[b] * t3[c];
                ge[1] += ph * t1[a] * d2[b] * t3[c];
                ge[2] += ph * t1[a] * t2[b] * d3[c];
                gw[0] += ph * (qi * d1[a] * t2[b] * t3[c] + e[0] * s1[a] * t2[b] * t3[c] + e[1] * d1[a] * d2[b] * t3[c] +
                               e[2] * d1[a] * t2[b] * d3[c]);
                gw[1] += ph * (qi * t1[a] * d2[b] * t3[c] + e[0] * d1[a] * d2[b] * t3[c] + e[1] * t1[a] * s2[b] * t3[c] +
                               e[2] * t1[a] * d2[b] * d3[c]);
                gw[2] += ph * (qi * t1[a] * t2[b] * d3[c] + e[0] * d1[a] * t2[b] * d3[c] + e[1] * t1[a] * d2[b] * d3[c] +
                               e[2] * t1[a] * t2[b] * s3[c]);
            }
    for (int b = 0; b < 3; ++b) {
        gd[b] = ge[0] * P->escale[b * 3 + 0] + ge[1] * P->escale[b * 3 + 1] + ge[2] * P->escale[b * 3 + 2];
        if (gr) gr[b] = gw[0] * P->escale[b * 3 + 0] + gw[1] * P->escale[b * 3 + 1] + gw[2] * P->escale[b * 3 + 2];
    }
}

/* Influence part of the reciprocal virial: sum_m |F|^2 G [-delta_ab + 2 m*_a m*_b (pi^2/beta^2 +
 * 1/|m*|^2)] (strain derivative of pme.py:243-267 at fixed fractional coordinates).  Needs the
 * forward transform: called on a fresh spread. */
static void pme_influence_virial(pme_t *P, const double *q, const double *d, int n, double W[9]) {
    pme_spread(P, q, d, n);
    fft3d(P->grid, P->K, -1, 0);
    int K0 = P->K[0], K1 = P->K[1], K2 = P->K[2];
    double acc[9] = {0};
    for (int i = 0; i < K0; ++i)
        for (int j = 0; j < K1; ++j)
            for (int k = 0; k < K2; ++k) {
                size_t id = ((size_t)i * K1 + j) * K2 + k;
                if (P->G[id] == 0.0) continue;
                int m[3] = {i <= (K0 - 1) / 2 ? i : i - K0, j <= (K1 - 1) / 2 ? j : j - K1,
                            k <= (K2 - 1) / 2 ? k : k - K2};
                if (K0 % 2 == 0 && i == K0 / 2) m[0] = -K0 / 2;
                if (K1 % 2 == 0 && j == K1 / 2) m[1] = -K1 / 2;
                if (K2 % 2 == 0 && k == K2 / 2) m[2] = -K2 / 2;
                double mv[3];
                for (int c = 0; c < 3; ++c)
                    mv[c] = m[0] * P->Hinv[c * 3 + 0] + m[1] * P->Hinv[c * 3 + 1] + m[2] * P->Hinv[c * 3 + 2];
                double msq = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
                double complex F = P->grid[id];
                double e2 = P->G[id] * (creal(F) * creal(F) + cimag(F) * cimag(F));
                double fac = 2.0 * (M_PI * M_PI / (P->beta * P->beta) + 1.0 / msq);
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) acc[a * 3 + b] += e2 * ((a == b ? -1.0 : 0.0) + fac * mv[a] * mv[b]);
            }
    for (int k = 0; k < 9; ++k) W[k] += acc[k];
}

/* ------------------------------------------------------------------ pair rows (forcefield.py:1140-1195) */
typedef struct {
    long long *start;   /* (n + 1) */
    int *k;
    double *x;          /* (pairs, 3) x_i - x_k, minimum image */
    double *G;          /* (pairs, 4) */
    double *wv;         /* van der Waals weight: 0 intramolecular, 1 otherwise */
    unsigned char *we;  /* 1: inside the electrostatics cutoff (split rows, forcefield.py:1197-1238) */
} rows_t;

static int *atom_mol(const pgmo_system *sys) {
    int *m = malloc(sizeof(int) * sys->n);
    for (int a = 0; a < sys->nmol; ++a)
        for (int i = sys->mol_start[a]; i < sys->mol_start[a + 1]; ++i) m[i] = a;
    return m;
}

/* Candidate partners of atoms: the atoms of the 27 cells around an atom's cell in fractional
 * coordinates, cells at least one cutoff high across their planes (the grid has at least 3 cells
 * along every axis; otherwise every atom is a candidate).  A pair inside the cutoff under the
 * minimum image has an image whose fractional separation is below rc / h_a along every axis
 * (h_a the box height across the planes of axis a), so it lies in a neighbouring cell. */
typedef struct {
    int nc[3];
    int *start, *atoms, *cell;  /* (cells + 1), (n) atoms by cell in index order, (n) cell of each atom */
} cells_t;

static int cells_init(cells_t *L, const double *pos, const double *H, int n, double rc) {
    double Hi[9];
    inv3(H, Hi);
    long long ncell = 1;
    for (int a = 0; a < 3; ++a) {
        double h = 1.0 / sqrt(Hi[0 * 3 + a] * Hi[0 * 3 + a] + Hi[1 * 3 + a] * Hi[1 * 3 + a] + Hi[2 * 3 + a] * Hi[2 * 3 + a]);
        L->nc[a] = (int)floor(h / rc);
        if (L->nc[a] < 3 || n < 4096) return 0;
        if (L->nc[a] > 256) L->nc[a] = 256;
        ncell *= L->nc[a];
    }
    L->cell = malloc(sizeof(int) * n);
    L->start = calloc(ncell + 1, sizeof(int));
    L->atoms = malloc(sizeof(int) * n);
    for (int i = 0; i < n; ++i) {
        int c[3];
        for (int a = 0; a < 3; ++a) {
            double u = pos[i * 3] * Hi[a] + pos[i * 3 + 1] * Hi[3 + a] + pos[i * 3 + 2] * Hi[6 + a];
            c[a] = (int)floor((u - floor(u)) * L->nc[a]);
            if (c[a] >= L->nc[a]) c[a] = L->nc[a] - 1;
            if (c[a] < 0) c[a] = 0;
        }
        L->cell[i] = (c[0] * L->nc[1] + c[1]) * L->nc[2] + c[2];
        L->start[L->cell[i] + 1]++;
    }
    for (long long c = 0; c < ncell; ++c) L->start[c + 1] += L->start[c];
    int *fill = malloc(sizeof(int) * ncell);
    memcpy(fill, L->start, sizeof(int) * ncell);
    for (int i = 0; i < n; ++i) L->atoms[fill[L->cell[i]]++] = i;
    free(fill);
    return 1;
}

static int cmp_int(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* The candidates of atom i in ascending index order (i itself excluded); returns their number. */
static int candidates(const cells_t *L, int use_cells, int n, int i, int *out) {
    int m = 0;
    if (!use_cells) {
        for (int k = 0; k < n; ++k)
            if (k != i) out[m++] = k;
        return m;
    }
    int c = L->cell[i];
    int c2 = c % L->nc[2], c1 = (c / L->nc[2]) % L->nc[1], c0 = c / (L->nc[1] * L->nc[2]);
    for (int d0 = -1; d0 <= 1; ++d0)
        for (int d1 = -1; d1 <= 1; ++d1)
            for (int d2 = -1; d2 <= 1; ++d2) {
                int e0 = (c0 + d0 + L->nc[0]) % L->nc[0], e1 = (c1 + d1 + L->nc[1]) % L->nc[1],
                    e2 = (c2 + d2 + L->nc[2]) % L->nc[2];
                int cc = (e0 * L->nc[1] + e1) * L->nc[2] + e2;
                for (int t = L->start[cc]; t < L->start[cc + 1]; ++t)
                    if (L->atoms[t] != i) out[m++] = L->atoms[t];
            }
    qsort(out, m, sizeof(int), cmp_int);
    return m;
}

/* Every atom's row: its molecule partners (the rigid special table, topology.py:161-178, vdW
 * weight 0) then every other atom inside the cutoff (vdW weight 1), all masked to r < rc. */
static void build_rows(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H,
                       rows_t *R) {
    int n = sys->n;
    int *mol = atom_mol(sys);
    double rc2 = s->cutoff * s->cutoff;
    cells_t L;
    int use_cells = cells_init(&L, pos, H, n, s->cutoff);
    int maxc = n;
    if (use_cells) {  /* the largest 27-cell neighbourhood */
        maxc = 0;
        for (int i = 0; i < n; ++i) {
            int c = L.cell[i], m = 0;
            int c2 = c % L.nc[2], c1 = (c / L.nc[2]) % L.nc[1], c0 = c / (L.nc[1] * L.nc[2]);
            for (int d0 = -1; d0 <= 1; ++d0)
                for (int d1 = -1; d1 <= 1; ++d1)
                    for (int d2 = -1; d2 <= 1; ++d2) {
                        int cc = (((c0 + d0 + L.nc[0]) % L.nc[0]) * L.nc[1] + (c1 + d1 + L.nc[1]) % L.nc[1]) * L.nc[2] +
                                 (c2 + d2 + L.nc[2]) % L.nc[2];
                        m += L.start[cc + 1] - L.start[cc];
                    }
            if (m > maxc) maxc = m;
        }
    }
    R->start = calloc(n + 1, sizeof(long long));
    int *cnt = calloc(n, sizeof(int));
#pragma omp parallel
    {
        int *cand = malloc(sizeof(int) * (maxc + 1));
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i) {
            int nc = candidates(&L, use_cells, n, i, cand), c = 0;
            for (int t = 0; t < nc; ++t) {
                int k = cand[t];
                double x[3] = {pos[i * 3] - pos[k * 3], pos[i * 3 + 1] - pos[k * 3 + 1], pos[i * 3 + 2] - pos[k * 3 + 2]};
                min_image(x, H);
                if (x[0] * x[0] + x[1] * x[1] + x[2] * x[2] < rc2) ++c;
            }
            cnt[i] = c;
        }
        free(cand);
    }
    for (int i = 0; i < n; ++i) R->start[i + 1] = R->start[i] + cnt[i];
    long long np = R->start[n];
    R->k = malloc(sizeof(int) * (np ? np : 1));
    R->x = malloc(sizeof(double) * 3 * (np ? np : 1));
    R->G = malloc(sizeof(double) * 4 * (np ? np : 1));
    R->wv = malloc(sizeof(double) * (np ? np : 1));
    R->we = malloc(np ? np : 1);
    const double rce = (s->elec_cutoff > 0.0 && s->elec_cutoff < s->cutoff) ? s->elec_cutoff : s->cutoff;
    const double rce2 = rce * rce;
#pragma omp parallel
    {
        int *cand = malloc(sizeof(int) * (maxc + 1));
#pragma omp for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i) {
            long long o = R->start[i];
            int mi = mol[i];
            int nc = candidates(&L, use_cells, n, i, cand);
            /* specials first (same molecule, sorted), then the others in index order */
            for (int pass = 0; pass < 2; ++pass)
                for (int t = 0; t < nc; ++t) {
                    int k = cand[t];
                    if ((mol[k] == mi) != (pass == 0)) continue;
                    double x[3] = {pos[i * 3] - pos[k * 3], pos[i * 3 + 1] - pos[k * 3 + 1], pos[i * 3 + 2] - pos[k * 3 + 2]};
                    min_image(x, H);
                    double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                    if (r2 >= rc2) continue;
                    R->k[o] = k;
                    memcpy(R->x + 3 * o, x, sizeof(x));
                    double a = 1.0 / sqrt(2.0 * (sys->radius[i] * sys->radius[i] + sys->radius[k] * sys->radius[k]));
                    pair_kernels(a, s->beta, sqrt(r2), R->G + 4 * o);
                    R->wv[o] = pass == 0 ? 0.0 : 1.0;
                    R->we[o] = r2 < rce2;
                    ++o;
                }
        }
        free(cand);
    }
    if (use_cells) {
        free(L.cell);
        free(L.start);
        free(L.atoms);
    }
    free(cnt);
    free(mol);
}

static void free_rows(rows_t *R) {
    free(R->start);
    free(R->k);
    free(R->x);
    free(R->G);
    free(R->wv);
    free(R->we);
}

/* sum_k de_ik/dd_i (forcefield.py:1395-1402), q may be NULL. */
static void row_field(const rows_t *R, int n, const double *q, const double *d, double *out) {
#pragma omp parallel for schedule(dynamic, 32)
    for (int i = 0; i < n; ++i) {
        double f[3] = {0, 0, 0};
        for (long long o = R->start[i]; o < R->start[i + 1]; ++o) {
            if (!R->we[o]) continue;
            int k = R->k[o];
            const double *x = R->x + 3 * o, *G = R->G + 4 * o, *dk = d + 3 * k;
            double dkx = dk[0] * x[0] + dk[1] * x[1] + dk[2] * x[2];
            double c = -G[2] * dkx - (q ? q[k] * G[1] : 0.0);
            for (int j = 0; j < 3; ++j) f[j] += c * x[j] + G[1] * dk[j];
        }
        memcpy(out + 3 * i, f, sizeof(f));
    }
}

/* ------------------------------------------------------------------ permanent dipoles */
void perm_dipoles_impl(const pgmo_system *sys, const double *pos, const double *H, double *p) {
    memset(p, 0, sizeof(double) * 3 * sys->n);
    for (int m = 0; m < sys->ncov; ++m) {
        int i = sys->cov_i[m], j = sys->cov_j[m];
        double v[3] = {pos[j * 3] - pos[i * 3], pos[j * 3 + 1] - pos[i * 3 + 1], pos[j * 3 + 2] - pos[i * 3 + 2]};
        min_image(v, H);
        double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (int a = 0; a < 3; ++a) p[i * 3 + a] += sys->cov_c[m] * v[a] / l;
    }
}

int pgmo_perm_dipoles(const pgmo_system *sys, const double *pos, const double *H, double *p) {
    perm_dipoles_impl(sys, pos, H, p);
    return 0;
}

/* ------------------------------------------------------------------ context */
typedef struct {
    const pgmo_system *sys;
    const pgmo_settings *s;
    rows_t R;
    pme_t P;
    double c_self;
    double *tmp, *tmp2;
} ctx_t;

static void ctx_init(ctx_t *C, const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H) {
    C->sys = sys;
    C->s = s;
    build_rows(sys, s, pos, H, &C->R);
    pme_init(&C->P, s, H, sys->n);
    pme_setup(&C->P, pos, sys->n);
    C->c_self = 4.0 * s->beta * s->beta * s->beta / (3.0 * SQRT_PI);
    C->tmp = malloc(sizeof(double) * 3 * sys->n);
    C->tmp2 = malloc(sizeof(double) * 3 * sys->n);
}

static void ctx_free(ctx_t *C) {
    free_rows(&C->R);
    pme_free(&C->P);
    free(C->tmp);
    free(C->tmp2);
}

/* Total field -dU/dd = -(row field + dU_rec/dd - c_self d) (forcefield.py:1428-1433). */
static void field(ctx_t *C, const double *q, const double *d, double *out) {
    int n = C->sys->n;
    row_field(&C->R, n, q, d, C->tmp);
    pme_energy_phi(&C->P, q, d, n);
#pragma omp parallel for
    for (int i = 0; i < n; ++i) {
        double gd[3];
        pme_gather(&C->P, i, q ? q[i] : 0.0, d + 3 * i, gd, NULL);
        for (int a = 0; a < 3; ++a) out[3 * i + a] = -(C->tmp[3 * i + a] + gd[a] - C->c_self * d[3 * i + a]);
    }
}

/* A v = v / alpha - field(0, v) (forcefield.py:1694-1712). */
static void apply_A(ctx_t *C, const double *v, double *out) {
    int n = C->sys->n;
    double *f = malloc(sizeof(double) * 3 * n);
    field(C, NULL, v, f);
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) out[3 * i + a] = v[3 * i + a] / C->sys->alpha[i] - f[3 * i + a];
    free(f);
}

static double dot(const double *a, const double *b, int m) {
    double s = 0.0;
    for (int i = 0; i < m; ++i) s += a[i] * b[i];
    return s;
}

/* The short-range operator of the local preconditioner: A_loc v = v / alpha + the row field of v over
 * the electrostatic row entries closer than local_cut (forcefield.py:1771-1772). */
static void apply_A_loc(ctx_t *C, const double *v, double *out) {
    const rows_t *R = &C->R;
    int n = C->sys->n;
    const double lc2 = C->s->local_cut * C->s->local_cut;
#pragma omp parallel for schedule(dynamic, 32)
    for (int i = 0; i < n; ++i) {
        double f[3] = {0, 0, 0};
        for (long long o = R->start[i]; o < R->start[i + 1]; ++o) {
            const double *x = R->x + 3 * o;
            if (!R->we[o] || x[0] * x[0] + x[1] * x[1] + x[2] * x[2] >= lc2) continue;
            const double *G = R->G + 4 * o, *dk = v + 3 * R->k[o];
            double dkx = dk[0] * x[0] + dk[1] * x[1] + dk[2] * x[2];
            for (int j = 0; j < 3; ++j) f[j] += -G[2] * dkx * x[j] + G[1] * dk[j];
        }
        for (int j = 0; j < 3; ++j) out[3 * i + j] = v[3 * i + j] / C->sys->alpha[i] + f[j];
    }
}

/* z = M^-1 r: Jacobi z = alpha r, refined with local_niter > 0 by that many inner CG iterations on
 * A_loc from z (forcefield.py:1766-1792). */
static void precond(ctx_t *C, const double *r, double *z) {
    int n = C->sys->n, m = 3 * n;
    const double *al = C->sys->alpha;
    for (int i = 0; i < m; ++i) z[i] = al[i / 3] * r[i];
    if (C->s->local_niter <= 0) return;
    double *rr = malloc(sizeof(double) * m), *p = malloc(sizeof(double) * m), *Ap = malloc(sizeof(double) * m);
    apply_A_loc(C, z, Ap);
    for (int i = 0; i < m; ++i) {
        rr[i] = r[i] - Ap[i];
        p[i] = al[i / 3] * rr[i];
    }
    double rz = dot(rr, p, m);
    for (int it = 0; it < C->s->local_niter; ++it) {
        apply_A_loc(C, p, Ap);
        double a = rz / fmax(dot(p, Ap, m), 1e-300), rzn = 0.0;
        for (int i = 0; i < m; ++i) {
            z[i] += a * p[i];
            rr[i] -= a * Ap[i];
            rzn += rr[i] * al[i / 3] * rr[i];
        }
        double b = rzn / fmax(rz, 1e-300);
        for (int i = 0; i < m; ++i) p[i] = al[i / 3] * rr[i] + b * p[i];
        rz = rzn;
    }
    free(rr);
    free(p);
    free(Ap);
}

/* PCG (Jacobi, or the local preconditioner: flexible) with the Polak-Ribiere beta, pmemd-pgm's
 * max-norm test and the peek step (forcefield.py:1714-1821). */
static void cg_to(ctx_t *C, double *x, double *r, double norm, double tol, int max_iter, int *iters, double *resid) {
    const pgmo_settings *s = C->s;
    int n = C->sys->n, m = 3 * n;
    const double *al = C->sys->alpha;
    double *z = malloc(sizeof(double) * m), *p = malloc(sizeof(double) * m), *Ap = malloc(sizeof(double) * m),
           *rn = malloc(sizeof(double) * m);
    precond(C, r, z);
    memcpy(p, z, sizeof(double) * m);
    double rz = dot(r, z, m);
    double err = 0.0;
    for (int i = 0; i < m; ++i) err = fmax(err, fabs(al[i / 3] * r[i]));
    err /= norm;
    int it = 0;
    while (err > tol && it < max_iter) {
        apply_A(C, p, Ap);
        double pAp = dot(p, Ap, m);
        double a = rz / fmax(pAp, 1e-300);
        for (int i = 0; i < m; ++i) {
            x[i] += a * p[i];
            rn[i] = r[i] - a * Ap[i];
        }
        double num = 0.0, rzn = 0.0;
        err = 0.0;
        precond(C, rn, z);
        for (int i = 0; i < m; ++i) {
            num += z[i] * (rn[i] - r[i]);
            rzn += rn[i] * z[i];
            err = fmax(err, fabs(al[i / 3] * rn[i]));
        }
        err /= norm;
        double beta = num / fmax(rz, 1e-300);
        for (int i = 0; i < m; ++i) p[i] = z[i] + beta * p[i];
        memcpy(r, rn, sizeof(double) * m);
        rz = rzn;
        ++it;
    }
    if (s->peek != 0.0)
        for (int i = 0; i < m; ++i) x[i] += s->peek * r[i] * al[i / 3];
    *iters = it;
    *resid = err;
    free(z);
    free(p);
    free(Ap);
    free(rn);
}

static void cg(ctx_t *C, double *x, double *r, double norm, int *iters, double *resid) {
    cg_to(C, x, r, norm, C->s->tol, C->s->max_iter, iters, resid);
}

/* Initial guess and residual, fused or plain, then CG; pushes the history (forcefield.py:1917-2008). */
static void solve(ctx_t *C, const double *q, const double *pdip, double *mu, double *hist, int *count, double *normp,
                  int *iters, double *resid) {
    const pgmo_settings *s = C->s;
    int n = C->sys->n, m = 3 * n;
    const double *al = C->sys->alpha;
    double *x0 = calloc(m, sizeof(double)), *r0 = malloc(sizeof(double) * m), *b = malloc(sizeof(double) * m),
           *dd = malloc(sizeof(double) * m), *Ax = malloc(sizeof(double) * m);
    /* mu3 / mu4 extrapolations (forcefield.py:605); predictor 1 = the previous step's dipoles */
    static const double c4[4] = {4.0, -6.0, 4.0, -1.0}, c3[3] = {3.0, -3.0, 1.0}, c1[1] = {1.0};
    int K = s->predictor == 4 ? 4 : (s->predictor == 3 ? 3 : (s->predictor == 1 ? 1 : 0));
    const double *cc = K == 4 ? c4 : (K == 3 ? c3 : c1);
    int have = K > 0 && *count >= K;
    if (have)
        for (int j = 0; j < K; ++j)
            for (int i = 0; i < m; ++i) x0[i] += cc[j] * hist[(size_t)j * m + i];
    double norm;
    if (K > 0 && s->fused && have && (*count % s->norm_refresh) != 0) {
        for (int i = 0; i < m; ++i) dd[i] = pdip[i] + x0[i];
        field(C, q, dd, r0);
        for (int i = 0; i < m; ++i) r0[i] -= x0[i] / al[i / 3];
        norm = *normp;
    } else {
        field(C, q, pdip, b);
        double sab = 0.0;
        for (int i = 0; i < m; ++i) sab += fabs(al[i / 3] * b[i]);
        if (!have)
            for (int i = 0; i < m; ++i) x0[i] = al[i / 3] * b[i];
        apply_A(C, x0, Ax);
        for (int i = 0; i < m; ++i) r0[i] = b[i] - Ax[i];
        norm = sab / m + 1e-300;
    }
    cg(C, x0, r0, norm, iters, resid);
    memcpy(mu, x0, sizeof(double) * m);
    memmove(hist + m, hist, sizeof(double) * 3 * m);
    memcpy(hist, mu, sizeof(double) * m);
    *count += 1;
    *normp = norm;
    free(x0);
    free(r0);
    free(b);
    free(dd);
    free(Ax);
}

/* Amber vdwmeth=1 tail (lj.py:87-114). */
static double lj_tail(const pgmo_system *sys, double vol, double rc) {
    double M[7] = {0};
    for (int i = 0; i < sys->n; ++i) {
        double pw = 1.0;
        for (int k = 0; k < 7; ++k) {
            M[k] += sys->sqrt_eps[i] * pw;
            pw *= sys->rmin_half[i];
        }
    }
    static const double binom[7] = {1, 6, 15, 20, 15, 6, 1};
    double SB = 0.0;
    for (int k = 0; k < 7; ++k) SB += binom[k] * M[k] * M[6 - k];
    SB *= 2.0;
    return -2.0 * M_PI * SB / (3.0 * vol * rc * rc * rc);
}

/* Offsets of every atom from its molecule's centre of mass, molecule made whole from its first atom. */
static void com_offsets(const pgmo_system *sys, const double *pos, const double *H, double *off) {
    for (int a = 0; a < sys->nmol; ++a) {
        int i0 = sys->mol_start[a], i1 = sys->mol_start[a + 1];
        double c[3] = {0, 0, 0}, mt = 0.0;
        for (int i = i0; i < i1; ++i) {
            double v[3] = {pos[i * 3] - pos[i0 * 3], pos[i * 3 + 1] - pos[i0 * 3 + 1], pos[i * 3 + 2] - pos[i0 * 3 + 2]};
            min_image(v, H);
            memcpy(off + 3 * i, v, sizeof(v));
            for (int k = 0; k < 3; ++k) c[k] += sys->mass[i] * v[k];
            mt += sys->mass[i];
        }
        for (int i = i0; i < i1; ++i)
            for (int k = 0; k < 3; ++k) off[3 * i + k] -= c[k] / mt;
    }
}

/* Energies, forces and molecular virial at fixed mu: the row terms (forcefield.py:2294-2360), the
 * non-pair terms (2011-2045), the covalent-frame pull-back (2362-2430), the strain derivative of the
 * same energy (608-662, 2628-2695) written out analytically. */
static void energy_forces(ctx_t *C, const double *pos, const double *H, const double *mu, const double *pdip,
                          double *forces, pgmo_result *res, const double *delta, const int *blk, double keep_blk) {
    const pgmo_system *sys = C->sys;
    const pgmo_settings *s = C->s;
    int n = sys->n;
    double *d = malloc(sizeof(double) * 3 * n), *dEdd = malloc(sizeof(double) * 3 * n),
           *off = malloc(sizeof(double) * 3 * n);
    for (int i = 0; i < 3 * n; ++i) d[i] = pdip[i] + mu[i];
    com_offsets(sys, pos, H, off);
    double se = 0.0, sl = 0.0, W[9] = {0};
#pragma omp parallel
    {
        double se_t = 0.0, sl_t = 0.0, W_t[9] = {0};
#pragma omp for schedule(dynamic, 32)
        for (int i = 0; i < n; ++i) {
            double gx[3] = {0, 0, 0}, gl[3] = {0, 0, 0}, fd[3] = {0, 0, 0};
            const double *di = d + 3 * i;
            double qi = sys->q[i];
            for (long long o = C->R.start[i]; o < C->R.start[i + 1]; ++o) {
                int k = C->R.k[o];
                const double *x = C->R.x + 3 * o, *dk = d + 3 * k;
                /* beyond the electrostatics cutoff only the van der Waals term (split rows) */
                const double G0[4] = {0, 0, 0, 0}, *G = C->R.we[o] ? C->R.G + 4 * o : G0;
                double qk = sys->q[k];
                double dix = di[0] * x[0] + di[1] * x[1] + di[2] * x[2];
                double dkx = dk[0] * x[0] + dk[1] * x[1] + dk[2] * x[2];
                double didk = di[0] * dk[0] + di[1] * dk[1] + di[2] * dk[2];
                double t = qi * dkx - qk * dix;
                double e = qi * qk * G[0] + t * G[1] - G[2] * dix * dkx + G[1] * didk;
                double radial = -qi * qk * G[1] - t * G[2] + G[3] * dix * dkx - G[2] * didk;
                double g[3];
                for (int j = 0; j < 3; ++j) {
                    double cross = di[j] * dkx + dk[j] * dix;
                    g[j] = radial * x[j] + qi * G[1] * dk[j] - qk * G[1] * di[j] - G[2] * cross;
                    gx[j] += g[j];
                }
                if (delta) {
                    /* iEL/0-SCF shadow energy: minus the pair terms of the dipoles delta alone
                     * (forcefield.py:2316-2330); inside a preconditioner block scaled by 1 - 1/omega */
                    double w = (blk && blk[i] >= 0 && blk[i] == blk[k]) ? keep_blk : 1.0;
                    const double Di[3] = {w * delta[3 * i], w * delta[3 * i + 1], w * delta[3 * i + 2]};
                    const double *Dk = delta + 3 * k;
                    double Dix = Di[0] * x[0] + Di[1] * x[1] + Di[2] * x[2];
                    double Dkx = Dk[0] * x[0] + Dk[1] * x[1] + Dk[2] * x[2];
                    double DiDk = Di[0] * Dk[0] + Di[1] * Dk[1] + Di[2] * Dk[2];
                    e += G[2] * Dix * Dkx - G[1] * DiDk;
                    double rad2 = -G[3] * Dix * Dkx + G[2] * DiDk;
                    for (int j = 0; j < 3; ++j) gx[j] += rad2 * x[j] + G[2] * (Di[j] * Dkx + Dk[j] * Dix);
                }
                se_t += e;
                double c = -qk * G[1] - G[2] * dkx;
                for (int j = 0; j < 3; ++j) fd[j] += c * x[j] + G[1] * dk[j];
                double gv[3] = {0, 0, 0};
                if (s->lj && C->R.wv[o] != 0.0) {
                    double rm = sys->rmin_half[i] + sys->rmin_half[k];
                    double ep = sys->sqrt_eps[i] * sys->sqrt_eps[k];
                    double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
                    double s2 = rm * rm / r2, s6 = s2 * s2 * s2;
                    double wv = C->R.wv[o];
                    sl_t += wv * ep * (s6 * s6 - 2.0 * s6);
                    double dl = wv * ep * 12.0 * (s6 - s6 * s6) / r2;
                    for (int j = 0; j < 3; ++j) {
                        gv[j] = dl * x[j];
                        gl[j] += gv[j];
                    }
                }
                /* strain: x_ik -> x_ik + eps y, y = x_ik - off_i + off_k (molecular scaling) */
                double y[3];
                for (int j = 0; j < 3; ++j) y[j] = x[j] - off[3 * i + j] + off[3 * k + j];
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) W_t[a * 3 + b] += 0.5 * (KE * g[a] + gv[a]) * y[b];
            }
            for (int j = 0; j < 3; ++j) {
                forces[3 * i + j] = -(KE * gx[j] + gl[j]);
                dEdd[3 * i + j] = KE * fd[j];
            }
        }
#pragma omp critical
        {
            se += se_t;
            sl += sl_t;
            for (int k = 0; k < 9; ++k) W[k] += W_t[k];
        }
    }
    /* reciprocal space: energy, phi, per-atom gradients */
    double Erec = pme_energy_phi(&C->P, sys->q, d, n);
    double Wr[9] = {0};
#pragma omp parallel
    {
        double Wt[9] = {0};
#pragma omp for
        for (int i = 0; i < n; ++i) {
            double gd[3], gr[3];
            pme_gather(&C->P, i, sys->q[i], d + 3 * i, gd, gr);
            for (int j = 0; j < 3; ++j) {
                forces[3 * i + j] -= KE * gr[j];
                dEdd[3 * i + j] += KE * (gd[j] - C->c_self * d[3 * i + j]);
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    Wt[a * 3 + b] -= KE * (gr[a] * off[3 * i + b] + gd[a] * d[3 * i + b]);
        }
#pragma omp critical
        for (int k = 0; k < 9; ++k) Wr[k] += Wt[k];
    }
    double Wi[9] = {0};
    pme_influence_virial(&C->P, sys->q, d, n, Wi);
    for (int k = 0; k < 9; ++k) W[k] += Wr[k] + KE * Wi[k];
    /* shadow energy: minus the reciprocal energy of delta alone; its position gradient at fixed delta
     * (the strain derivative stays the fixed-mu one of strain_derivative, forcefield.py:2628) */
    double Erec_d = 0.0;
    if (delta) {
        Erec_d = pme_energy_phi(&C->P, NULL, delta, n);
#pragma omp parallel for
        for (int i = 0; i < n; ++i) {
            double gd[3], gr[3];
            pme_gather(&C->P, i, 0.0, delta + 3 * i, gd, gr);
            for (int j = 0; j < 3; ++j) forces[3 * i + j] += KE * gr[j];
        }
    }
    /* covalent-dipole frames: p_i = sum c unit(r_j - r_i) pulled back (vjp of forcefield.py:1032-1042) */
    for (int m = 0; m < (s->perm ? sys->ncov : 0); ++m) {
        int i = sys->cov_i[m], j = sys->cov_j[m];
        double v[3] = {pos[j * 3] - pos[i * 3], pos[j * 3 + 1] - pos[i * 3 + 1], pos[j * 3 + 2] - pos[i * 3 + 2]};
        min_image(v, H);
        double l = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double u[3] = {v[0] / l, v[1] / l, v[2] / l};
        const double *g = dEdd + 3 * i;
        double ug = u[0] * g[0] + u[1] * g[1] + u[2] * g[2];
        for (int a = 0; a < 3; ++a) {
            double gv = sys->cov_c[m] * (g[a] - u[a] * ug) / l;
            forces[3 * j + a] -= gv;
            forces[3 * i + a] += gv;
        }
    }
    double q2 = 0.0, qs = 0.0, d2 = 0.0, upol = 0.0;
    for (int i = 0; i < n; ++i) {
        q2 += sys->q[i] * sys->q[i];
        qs += sys->q[i];
        d2 += d[3 * i] * d[3 * i] + d[3 * i + 1] * d[3 * i + 1] + d[3 * i + 2] * d[3 * i + 2];
        if (s->induce)
            for (int a = 0; a < 3; ++a) upol += mu[3 * i + a] * mu[3 * i + a] / (2.0 * sys->alpha[i]);
    }
    double vol = fabs(det3(H));
    double uself = -(s->beta / SQRT_PI) * q2 - 0.5 * C->c_self * d2;
    if (delta) { /* forcefield.py:2037-2042 */
        double dd2 = 0.0, dda = 0.0;
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a) {
                dd2 += delta[3 * i + a] * delta[3 * i + a];
                dda += delta[3 * i + a] * delta[3 * i + a] / (2.0 * sys->alpha[i]);
            }
        uself += 0.5 * C->c_self * dd2 - (1.0 - 1.0 / s->iel_omega) * dda;
    }
    double ubg = -M_PI * qs * qs / (2.0 * vol * s->beta * s->beta);
    double e_elec = 0.5 * KE * se + KE * (Erec - Erec_d + uself + ubg + upol);
    double tail = (s->lj && s->lj_lrc) ? lj_tail(sys, vol, s->cutoff) : 0.0;
    double e_vdw = 0.5 * sl + tail;
    for (int a = 0; a < 3; ++a) W[a * 3 + a] += -KE * ubg - 2.0 * tail;
    res->elec = e_elec;
    res->vdw = e_vdw;
    res->total = e_elec + e_vdw;
    memcpy(res->virial, W, sizeof(W));
    res->pairs = C->R.start[n];
    free(d);
    free(dEdd);
    free(off);
}

/* ------------------------------------------------------------------ extended-Lagrangian dipoles */
/* Dissipative extended-Lagrangian Verlet coefficients (kappa, a, c_0..c_K) of Niklasson et al.,
 * J. Chem. Phys. 130, 214109 (2009), the table of forcefield.py:667-676. */
static const struct {
    int K;
    double kappa, a;
    double c[10];
} XL[] = {
    {0, 1.0, 0.0, {0}},
    {3, 1.69, 0.150, {-2, 3, 0, -1}},
    {4, 1.75, 0.057, {-3, 6, -2, -2, 1}},
    {5, 1.82, 0.018, {-6, 14, -8, -3, 4, -1}},
    {6, 1.84, 0.0055, {-14, 36, -27, -2, 12, -6, 1}},
    {7, 1.86, 0.0016, {-36, 99, -88, 11, 32, -25, 8, -1}},
    {8, 1.88, 0.00044, {-99, 286, -286, 78, 78, -90, 42, -10, 1}},
    {9, 1.89, 0.00012, {-286, 858, -936, 364, 168, -300, 184, -63, 12, -1}},
};

static int xl_row(int order) {
    for (int r = 0; r < (int)(sizeof(XL) / sizeof(XL[0])); ++r)
        if (XL[r].K == order) return r;
    return -1;
}

/* Auxiliary dipoles kept: x_{n+1} and x_n ... x_{n-K} after a step, at least 3 (forcefield.py:1476-1479). */
int pgmo_iel_len(int order) {
    int nc = order == 0 ? 1 : order + 1;
    return nc + 1 > 3 ? nc + 1 : 3;
}

/* Block of every atom for the block preconditioner: molecules of 2..8 atoms (forcefield.py:1487-1517),
 * -1 elsewhere. */
static int *iel_blocks(const pgmo_system *sys) {
    int *b = malloc(sizeof(int) * sys->n);
    int nb = 0;
    for (int m = 0; m < sys->nmol; ++m) {
        int sz = sys->mol_start[m + 1] - sys->mol_start[m];
        int id = (sz >= 2 && sz <= 8) ? nb++ : -1;
        for (int i = sys->mol_start[m]; i < sys->mol_start[m + 1]; ++i) b[i] = id;
    }
    return b;
}

/* delta = M^-1 r per block, M = diag(1/alpha) + sum of the same-molecule row tensors G1 I - G2 x x^T
 * (forcefield.py:1530-1556), by Gaussian elimination with partial pivoting; alpha r outside blocks. */
static void block_solve(ctx_t *C, const int *blk, const double *r, double *d) {
    const pgmo_system *sys = C->sys;
#pragma omp parallel for schedule(dynamic, 16)
    for (int m = 0; m < sys->nmol; ++m) {
        int i0 = sys->mol_start[m], i1 = sys->mol_start[m + 1], nb = i1 - i0, N = 3 * nb;
        if (blk[i0] < 0) {
            for (int i = i0; i < i1; ++i)
                for (int a = 0; a < 3; ++a) d[3 * i + a] = sys->alpha[i] * r[3 * i + a];
            continue;
        }
        double M[24][25];
        for (int u = 0; u < N; ++u)
            for (int v = 0; v <= N; ++v) M[u][v] = 0.0;
        for (int i = i0; i < i1; ++i) {
            int li = i - i0;
            for (int a = 0; a < 3; ++a) {
                M[3 * li + a][3 * li + a] += 1.0 / sys->alpha[i];
                M[3 * li + a][N] = r[3 * i + a];
            }
            for (long long o = C->R.start[i]; o < C->R.start[i + 1]; ++o) {
                int k = C->R.k[o];
                if (k < i0 || k >= i1 || !C->R.we[o]) continue;
                const double *x = C->R.x + 3 * o, *G = C->R.G + 4 * o;
                int lk = k - i0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        M[3 * li + a][3 * lk + b] += (a == b ? G[1] : 0.0) - G[2] * x[a] * x[b];
            }
        }
        for (int c = 0; c < N; ++c) {
            int pr = c;
            for (int u = c + 1; u < N; ++u)
                if (fabs(M[u][c]) > fabs(M[pr][c])) pr = u;
            if (pr != c)
                for (int v = 0; v <= N; ++v) {
                    double t = M[c][v];
                    M[c][v] = M[pr][v];
                    M[pr][v] = t;
                }
            for (int u = c + 1; u < N; ++u) {
                double f = M[u][c] / M[c][c];
                for (int v = c; v <= N; ++v) M[u][v] -= f * M[c][v];
            }
        }
        for (int c = N - 1; c >= 0; --c) {
            double acc = M[c][N];
            for (int v = c + 1; v < N; ++v) acc -= M[c][v] * M[v][N];
            M[c][N] = acc / M[c][c];
        }
        for (int i = i0; i < i1; ++i)
            for (int a = 0; a < 3; ++a) d[3 * i + a] = M[3 * (i - i0) + a][N];
    }
}

/* One iEL step (forcefield.py:1558-1650): the warm-up steps solve to tol (from mu or alpha b on the
 * first, from x after), the others take x = xl[0] and either the 0-SCF update mu = x + omega delta,
 * delta = alpha r(x) or M^-1 r(x), r(x) = field(q, p + x) - x / alpha (one field sweep, no CG), or
 * ("scf") iel_iter CG iterations from x; then x_{n+1} = 2 x_n - x_{n-1} + kappa (mu - x_n)
 * + a sum_k c_k x_{n-k}.  delta_out: the shadow displacement (0 in the warm-up). */
static void solve_iel(ctx_t *C, const double *q, const double *pdip, const int *blk, double *mu, double *hist, int *count,
                      double *normp, double *xl, int *iters, double *resid, double *delta_out) {
    const pgmo_settings *s = C->s;
    int n = C->sys->n, m = 3 * n;
    const double *al = C->sys->alpha;
    int row = xl_row(s->iel_order);
    double kap = isnan(s->iel_kappa) ? XL[row].kappa : s->iel_kappa;
    double a = isnan(s->iel_alpha) ? XL[row].a : s->iel_alpha;
    int nc = s->iel_order == 0 ? 1 : s->iel_order + 1, K1 = pgmo_iel_len(s->iel_order);
    int first = *count == 0, warm = *count < (s->iel_order > 2 ? s->iel_order : 2) + 1;
    double *x = xl, *r0 = malloc(sizeof(double) * m), *b = malloc(sizeof(double) * m), *Ax = malloc(sizeof(double) * m),
           *dd = malloc(sizeof(double) * m), *d = calloc(m, sizeof(double));
    double norm;
    *iters = 0;
    if (warm) {
        field(C, q, pdip, b);
        double sab = 0.0;
        int any = 0;
        for (int i = 0; i < m; ++i) {
            sab += fabs(al[i / 3] * b[i]);
            any |= mu[i] != 0.0;
        }
        norm = sab / m + 1e-300;
        for (int i = 0; i < m; ++i) dd[i] = first ? (any ? mu[i] : al[i / 3] * b[i]) : x[i];
        apply_A(C, dd, Ax);
        for (int i = 0; i < m; ++i) r0[i] = b[i] - Ax[i];
        cg_to(C, dd, r0, norm, s->tol, s->max_iter, iters, resid);
        memcpy(mu, dd, sizeof(double) * m);
    } else {
        for (int i = 0; i < m; ++i) dd[i] = pdip[i] + x[i];
        field(C, q, dd, r0);
        for (int i = 0; i < m; ++i) r0[i] -= x[i] / al[i / 3];
        norm = *normp;
        if (s->iel == 1) {
            if (s->iel_precond == 1) block_solve(C, blk, r0, d);
            else
                for (int i = 0; i < m; ++i) d[i] = al[i / 3] * r0[i];
            double mx = 0.0;
            for (int i = 0; i < m; ++i) {
                d[i] *= s->iel_omega;
                mu[i] = x[i] + d[i];
                mx = fmax(mx, fabs(d[i]));
            }
            *resid = mx / norm;
        } else {
            memcpy(dd, x, sizeof(double) * m);
            int k = s->iel_iter;
            cg_to(C, dd, r0, norm, k > 0 ? 0.0 : s->tol, k > 0 ? k : s->max_iter, iters, resid);
            memcpy(mu, dd, sizeof(double) * m);
            for (int i = 0; i < m; ++i) d[i] = mu[i] - x[i];
        }
    }
    /* Xh: every entry mu on the first step, xl with xl[0] = mu in the warm-up, else xl */
    double *Xh = malloc(sizeof(double) * (size_t)K1 * m);
    for (int j = 0; j < K1; ++j)
        memcpy(Xh + (size_t)j * m, first ? mu : (j == 0 && warm ? mu : xl + (size_t)j * m), sizeof(double) * m);
    for (int i = 0; i < m; ++i) {
        double v = 2.0 * Xh[i] - Xh[m + i] + (warm ? 0.0 : kap * d[i]);
        if (a != 0.0)
            for (int k = 0; k < nc; ++k) v += a * XL[row].c[k] * Xh[(size_t)k * m + i];
        xl[i] = v;
    }
    for (int j = 1; j < K1; ++j) memcpy(xl + (size_t)j * m, Xh + (size_t)(j - 1) * m, sizeof(double) * m);
    memmove(hist + m, hist, sizeof(double) * 3 * m);
    memcpy(hist, mu, sizeof(double) * m);
    *count += 1;
    *normp = norm;
    for (int i = 0; i < m; ++i) delta_out[i] = (warm || s->iel != 1) ? 0.0 : d[i];
    free(Xh);
    free(r0);
    free(b);
    free(Ax);
    free(dd);
    free(d);
}

int pgmo_compute_iel(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H, double *mu,
                     double *hist, int *count, double *norm, double *xl, double *forces, pgmo_result *res) {
    if (xl_row(s->iel_order) < 0 || s->iel < 1 || s->iel > 2 || !(s->iel_omega > 0)) return 1;
    set_threads(s);
    ctx_t C;
    ctx_init(&C, sys, s, pos, H);
    int n = sys->n;
    double *p = calloc(3 * n, sizeof(double)), *delta = calloc(3 * n, sizeof(double));
    int *blk = s->iel_precond == 1 ? iel_blocks(sys) : NULL;
    if (s->perm) perm_dipoles_impl(sys, pos, H, p);
    res->iterations = 0;
    res->residual = 0.0;
    int shadow = 0;
    if (s->induce) {
        int warm = *count < (s->iel_order > 2 ? s->iel_order : 2) + 1;
        solve_iel(&C, sys->q, p, blk, mu, hist, count, norm, xl, &res->iterations, &res->residual, delta);
        shadow = s->iel == 1 && s->iel_shadow && !warm;
    } else {
        memset(mu, 0, sizeof(double) * 3 * n);
    }
    energy_forces(&C, pos, H, mu, p, forces, res, shadow ? delta : NULL, blk, 1.0 - 1.0 / s->iel_omega);
    free(p);
    free(delta);
    free(blk);
    ctx_free(&C);
    return 0;
}

static int set_threads(const pgmo_settings *s) {
#ifdef _OPENMP
    if (s->nthreads > 0) omp_set_num_threads(s->nthreads);
#endif
    (void)s;
    return 0;
}

int pgmo_compute(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H, double *mu,
                 double *hist, int *count, double *norm, double *forces, pgmo_result *res) {
    set_threads(s);
    ctx_t C;
    ctx_init(&C, sys, s, pos, H);
    int n = sys->n;
    double *p = calloc(3 * n, sizeof(double));
    if (s->perm) perm_dipoles_impl(sys, pos, H, p);
    res->iterations = 0;
    res->residual = 0.0;
    if (s->induce)
        solve(&C, sys->q, p, mu, hist, count, norm, &res->iterations, &res->residual);
    else
        memset(mu, 0, sizeof(double) * 3 * n);
    energy_forces(&C, pos, H, mu, p, forces, res, NULL, NULL, 1.0);
    free(p);
    ctx_free(&C);
    return 0;
}

int pgmo_energy_fixed_mu(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H,
                         const double *mu, double out[3]) {
    set_threads(s);
    ctx_t C;
    ctx_init(&C, sys, s, pos, H);
    int n = sys->n;
    double *p = calloc(3 * n, sizeof(double)), *f = malloc(sizeof(double) * 3 * n);
    if (s->perm) perm_dipoles_impl(sys, pos, H, p);
    pgmo_result r;
    energy_forces(&C, pos, H, mu, p, f, &r, NULL, NULL, 1.0);
    out[0] = r.elec;
    out[1] = r.vdw;
    out[2] = r.total;
    free(p);
    free(f);
    ctx_free(&C);
    return 0;
}

int pgmo_field(const pgmo_system *sys, const pgmo_settings *s, const double *pos, const double *H, const double *q,
               const double *d, double *out) {
    set_threads(s);
    ctx_t C;
    ctx_init(&C, sys, s, pos, H);
    field(&C, q, d, out);
    ctx_free(&C);
    return 0;
}
