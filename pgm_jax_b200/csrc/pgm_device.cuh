// pgm_device.cuh -- device helpers of the B200 pGM engine: types, per-system tables, minimum
// image, Gaussian-screened radial kernels, cardinal B-splines, warp/block reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgm {

constexpr double KE = 138.935458;  // kJ mol^-1 nm e^-2 (pgm_jax/units.py:31)
constexpr double SQRT_PI = 1.7724538509055160273;
constexpr double PI = 3.14159265358979323846;
constexpr int WARPS_PER_BLOCK = 8;       // warp-per-atom kernels: 8 atoms per block
constexpr int THREADS_PER_BLOCK = 256;   // thread-per-atom kernels: 256 atoms per block
constexpr int MAX_STAGES = 10;           // FFT stages per axis
constexpr int FFT_TILE = 16;             // lines per CTA in the strided FFT passes
constexpr int FFT_PAIRS = 8;             // complex lines (= 2x real lines) per CTA in the k3 pass
constexpr int FFT_THREADS = 256;         // threads per CTA of the FFT passes (<= the passes' launch bounds)

template <typename T> struct Vec4;
template <> struct Vec4<float> { using type = float4; };
template <> struct Vec4<double> { using type = double4; };
template <typename T> using v4 = typename Vec4<T>::type;

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };
template <typename T> using c2 = typename Cplx<T>::type;

__device__ __forceinline__ float t_erf(float x) { return erff(x); }
__device__ __forceinline__ double t_erf(double x) { return erf(x); }
__device__ __forceinline__ float t_exp(float x) { return expf(x); }
__device__ __forceinline__ double t_exp(double x) { return exp(x); }
__device__ __forceinline__ float t_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double t_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float t_rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ double t_rsqrt(double x) { return rsqrt(x); }

// Static description of one system of the batch (built on the host at creation).
struct SysInfo {
  int atom0, natom;     // atoms [atom0, atom0 + natom)
  int mol0, nmol;       // molecules
  int K[3], K3h;        // PME grid, K3/2 + 1
  long long rgrid0;     // offset of the real grids (elements)
  long long cgrid0;     // offset of the half-complex grids (elements)
  int nc[3];            // cell grid
  int cell0;            // offset of the cells
  int tw[3];            // offsets of the twiddle tables of K1, K2, K3
  int nst[3];           // FFT stages per axis
  int rad[3][MAX_STAGES];
  int mod0[3];          // offsets of the B-spline moduli of each axis
  double tail_sb;       // 2 sum_k C(6,k) M_k M_(6-k) of the LJ tail (lj.py:87-114)
  double sum_q, sum_q2; // charges
};

// Box-dependent values of one system, recomputed on the device every step from the caller's box.
struct BoxInfo {
  double H[9], Hinv[9], vol;
  double idiag[3];      // 1 / H_aa (minimum image by multiplication)
  double h[3];          // distances between lattice planes
  int R[3];             // cell search range of the candidate list (-1: whole axis)
  int changed;          // box differs from the previous step (influence function recomputed)
  int bad;              // not lower triangular or too small for the cutoff
};

// Per-system state of the conjugate-gradient solve, with the accumulators of its reductions.
struct CGSys {
  double rz, norm, err, beta, step;
  int it, active, have, fused, sweep2;
  int n3;               // 3 x atoms of the system (the mean of mean|alpha b|)
  double acc_pap, acc_rz, acc_num, acc_abs;
  unsigned long long acc_max;  // non-negative doubles compare as their bit patterns
  // learned guess: nn = this solve starts from x4 + the model's correction; fallback = its start
  // residual was worse than the record of the extrapolation's, so the solve restarts from x4.
  // Kept across solves: ref_err, the running mean of the extrapolation's start residual
  // max|alpha r0| / norm (plain starts, and every fallback), ref_n its samples, fallbacks the count.
  int nn, fallback, ref_n, pad_;
  double ref_err;
  long long fallbacks;
  // extended-Lagrangian dipoles: iel_ext = this step is an extended (0-SCF or SCF-from-x) step,
  // iel_first = the first step of the run; tol_s / maxit_s override the solver's tolerance and
  // iteration limit for this system (tol_s < 0, maxit_s < 0: the settings').
  int iel_ext, iel_first, maxit_s, pad2_;
  double tol_s;
  // local preconditioner: inner r.z (accumulated, and the next one), p.Ap, and beta of the inner CG
  double acc_lrz, acc_lrz2, acc_lpap, lb;
};

// Per-system accumulators of the energy pass.
struct EnergyAcc {
  double e_pair, e_lj, e_rec, d2, upol;
  double dd2, dda;      // iEL/0-SCF shadow energy: sum |delta|^2 and sum |delta|^2 / (2 alpha)
  double vir[9];        // pair + reciprocal (positional and dipolar) parts [kJ/mol]
  double vinf[7];       // influence-function part: E then xx, yy, zz, xy, xz, yz [e^2/nm]
};

// Sequential minimum image with the inverse diagonal precomputed (the row-build hot loop).
__device__ __forceinline__ void min_image_fast(double &x, double &y, double &z, const double *H, const double *id) {
  double n = rint(z * id[2]);
  x -= n * H[6]; y -= n * H[7]; z -= n * H[8];
  n = rint(y * id[1]);
  x -= n * H[3]; y -= n * H[4];
  n = rint(x * id[0]);
  x -= n * H[0];
}

// Sequential minimum image for a reduced lower-triangular box (pgm_jax/md/box.py:130-153).
__device__ __forceinline__ void min_image(double &x, double &y, double &z, const double *H) {
  double n = rint(z / H[8]);
  x -= n * H[6]; y -= n * H[7]; z -= n * H[8];
  n = rint(y / H[4]);
  x -= n * H[3]; y -= n * H[4];
  n = rint(x / H[0]);
  x -= n * H[0];
}

// B_0..B_3 of erf(a r)/r: Taylor series where (a r)^2 < 1, else the closed-form recursion
// (pgm_jax/md/kernels.py:76-118).  FP64 sums the reference's 15 terms; FP32 sums 11 (the terms
// m >= 11 are below 1/11! < 2.6e-8 of the first, under FP32 rounding).
// (The series divides by the odd integers 2m + 2n + 1 as multiplications by their reciprocals, and
// the closed form multiplies by 1/r: the same expressions, rounded once more per term.)
template <typename T>
__device__ __forceinline__ void erf_kernels(T a, T r, T B[4]) {
  const T x = a * r, s = x * x;
  const T c0 = T(2.0 / SQRT_PI) * a, a2x2 = T(2) * a * a;
  if (s < T(1)) {
    constexpr int NT = sizeof(T) == 4 ? 11 : 15;
    T t = T(1), acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
#pragma unroll
    for (int m = 0; m < NT; ++m) {
      acc0 += t * T(1.0 / (2 * m + 1));
      acc1 += t * T(1.0 / (2 * m + 3));
      acc2 += t * T(1.0 / (2 * m + 5));
      acc3 += t * T(1.0 / (2 * m + 7));
      t *= -s * T(1.0 / (m + 1));
    }
    B[0] = c0 * acc0;
    B[1] = c0 * a2x2 * acc1;
    B[2] = c0 * a2x2 * a2x2 * acc2;
    B[3] = c0 * a2x2 * a2x2 * a2x2 * acc3;
  } else if (s > (sizeof(T) == 4 ? T(30) : T(56))) {
    // far beyond the screening length: erf(a r) rounds to 1 and the terms of exp(-a^2 r^2), which
    // enter B_n with at most (2 a^2 r^2)^3 (2 a r / sqrt(pi)) / 15, stay below 1e-8 (FP32) or
    // 1e-18 (FP64) of it, so B_n are the bare Coulomb ones, (2n - 1)!! / r^(2n+1)
    const T ir = T(1) / r, ir2 = ir * ir;
    B[0] = ir;
    B[1] = B[0] * ir2;
    B[2] = T(3) * B[1] * ir2;
    B[3] = T(5) * B[2] * ir2;
  } else {
    const T ir = T(1) / r, ir2 = ir * ir;
    const T c = c0 * t_exp(-s);
    B[0] = t_erf(x) * ir;
    B[1] = (B[0] - c) * ir2;
    B[2] = (T(3) * B[1] - a2x2 * c) * ir2;
    B[3] = (T(5) * B[2] - a2x2 * a2x2 * c) * ir2;
  }
}

// Cardinal B-spline weights of order P at offset f, with first and second derivatives: the
// recursion of pgm_jax/md/pme.py:81-103 (theta[k] = M_P(f + P - 1 - k)).
template <typename T, int P, bool SECOND>
__device__ __forceinline__ void bspline(T f, T *th, T *dth, T *d2th) {
  T d[P], p1[P], p2[P];
#pragma unroll
  for (int k = 0; k < P; ++k) { d[k] = 0; p1[k] = 0; p2[k] = 0; }
  d[0] = T(1) - f;
  d[1] = f;
#pragma unroll
  for (int n = 3; n <= P; ++n) {
#pragma unroll
    for (int k = 0; k < P; ++k) { p2[k] = p1[k]; p1[k] = d[k]; }
    const T div = T(1) / T(n - 1);
    d[n - 1] = div * f * d[n - 2];
#pragma unroll
    for (int k = 1; k < n - 1; ++k) d[n - k - 1] = div * ((f + T(k)) * d[n - k - 2] + (T(n - k) - f) * d[n - k - 1]);
    d[0] = div * (T(1) - f) * d[0];
  }
#pragma unroll
  for (int k = 0; k < P; ++k) {
    th[k] = d[k];
    dth[k] = (k >= 1 ? p1[k - 1] : T(0)) - (k < P - 1 ? p1[k] : T(0));
    if (SECOND)
      d2th[k] = (k >= 2 ? p2[k - 2] : T(0)) - T(2) * ((k >= 1 && k - 1 < P - 2) ? p2[k - 1] : T(0)) +
                (k < P - 2 ? p2[k] : T(0));
  }
}

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may be
// scheduled as its predecessor in the stream drains (its blocks trigger the launch when they exit);
// it waits here for the predecessor's completion (its memory visible) before touching any data.
// Without the launch attribute the instruction is a no-op.
__device__ __forceinline__ void pdl_enter() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// Block of the batch -> (system, first atom of the block); blocks never straddle systems.
struct BlockMap {
  const int *sys;    // system of every block
  const int *atom0;  // first atom (global) of every block
};

}  // namespace pgm
