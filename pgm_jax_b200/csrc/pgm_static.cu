// pgm_static.cu -- the allocation-free field entry point (pgm_field_static).
//
// Some callers cannot allocate device memory: a jax.ffi custom call runs inside XLA, which has
// already reserved most of the GPU's memory for its own allocator and hands the call every buffer
// it may use, so a cudaMalloc there can fail or take memory XLA counts on; a call made while a
// stream is being captured into a CUDA graph may not call cudaMalloc at all.  pgm_field_static
// serves them: it computes the same total field -dU/dd as pgm_field (rows within the cutoff,
// smooth PME, self term) for ONE small system in FP64, with every intermediate (the PME grids and
// the box values) in the file-scope array g_field_scratch below instead of buffers of a handle.
//
// Pairs are taken by minimum image within the cutoff.  pgm_field's rows also keep every pair of
// atoms of one molecule, however far apart; the two agree for molecules smaller than the cutoff
// (water), and differ for a molecule whose atoms lie further apart than the cutoff.  The box must
// be the handle path's: lower triangular with a positive diagonal, the cutoff at most half of its
// smallest diagonal element; for any other box every field value is NaN (the box is on the device,
// so the check runs there).  The stream must belong to the current device.
//
// Limits (checked, PGM_ERR_UNSUPPORTED beyond them): at most PGM_STATIC_MAX_ATOMS atoms, mesh sizes
// K <= PGM_STATIC_MAX_K per axis with K1 K2 K3 <= PGM_STATIC_MAX_GRID points, spline order 4, 6 or 8.
// The array (2 complex FP64 grids + 64 doubles, 1 MB) is held by every GPU that loads the library
// until the process exits.  All calls share it and it keeps the last call's contents: each call
// clears the grid it accumulates into, and calls that overlap on the GPU (different streams or
// threads at the same time) race on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/pgm_b200.h"
#include "pgm_device.cuh"

namespace {

constexpr int SCR_BOX = 64;  // doubles at the end of the array: H, H^-1, volume, box flag
constexpr size_t SCR_DOUBLES = 4 * (size_t)PGM_STATIC_MAX_GRID + SCR_BOX;

// Grids A and B (complex, ping-pong of the 3D DFT) followed by the box block.
static __device__ __align__(256) double g_field_scratch[SCR_DOUBLES];

thread_local std::string g_static_err;
std::mutex g_static_mu;
double *g_static_ptr[64] = {nullptr};  // device address of g_field_scratch, per device

PgmStatus serr(PgmStatus s, const std::string &m) {
  g_static_err = m;
  return s;
}

struct StaticArgs {
  int n, K1, K2, K3;
  double cutoff, beta, c_self;
  const double *pos, *box, *q, *radius, *d;
  int with_q;
  double *field;
  double2 *A, *B;  // complex grids in the scratch array
  double *bx;      // box block: H (9), H^-1 (9), volume (1), unusable-box flag (1)
};

__global__ void ks_box_and_clear(StaticArgs s) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int ng = s.K1 * s.K2 * s.K3;
  for (int g = t; g < ng; g += gridDim.x * blockDim.x) s.A[g] = make_double2(0.0, 0.0);  // the spread accumulates here
  if (t == 0) {
    const double *H = s.box;
    double d = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) + H[2] * (H[3] * H[7] - H[4] * H[6]);
    double *Hi = s.bx + 9;
    Hi[0] = (H[4] * H[8] - H[5] * H[7]) / d; Hi[1] = (H[2] * H[7] - H[1] * H[8]) / d; Hi[2] = (H[1] * H[5] - H[2] * H[4]) / d;
    Hi[3] = (H[5] * H[6] - H[3] * H[8]) / d; Hi[4] = (H[0] * H[8] - H[2] * H[6]) / d; Hi[5] = (H[2] * H[3] - H[0] * H[5]) / d;
    Hi[6] = (H[3] * H[7] - H[4] * H[6]) / d; Hi[7] = (H[1] * H[6] - H[0] * H[7]) / d; Hi[8] = (H[0] * H[4] - H[1] * H[3]) / d;
    for (int k = 0; k < 9; ++k) s.bx[k] = H[k];
    s.bx[18] = fabs(d);
    // the minimum image below needs the handle path's box: lower triangular, positive diagonal,
    // the cutoff at most half the smallest diagonal element; otherwise the field is NaN
    int bad = (fabs(H[1]) > 1e-12 * fabs(H[0])) || (fabs(H[2]) > 1e-12 * fabs(H[0])) ||
              (fabs(H[5]) > 1e-12 * fabs(H[0])) || !(H[0] > 0 && H[4] > 0 && H[8] > 0) ||
              !(s.cutoff <= 0.5 * fmin(H[0], fmin(H[4], H[8])));
    s.bx[19] = bad ? 1.0 : 0.0;
  }
}

template <int P>
__device__ void ks_spline(const StaticArgs &s, int i, int b[3], double th[3][P], double dth[3][P]) {
  const double *Hi = s.bx + 9;
  const int K[3] = {s.K1, s.K2, s.K3};
  for (int ax = 0; ax < 3; ++ax) {
    double u = s.pos[3 * i] * Hi[0 * 3 + ax] + s.pos[3 * i + 1] * Hi[1 * 3 + ax] + s.pos[3 * i + 2] * Hi[2 * 3 + ax];
    double fr = u - floor(u);
    if (!(fr >= 0.0 && fr < 1.0)) fr = 0.0;
    double w = fr * K[ax], fl = floor(w);
    int bv = (int)fl;
    if (bv >= K[ax]) bv -= K[ax];
    if (bv < 0) bv = 0;
    b[ax] = bv;
    pgm::bspline<double, P, false>(w - fl, th[ax], dth[ax], nullptr);
  }
}

// Charges and dipoles spread on grid A (pme.py:306-337).
template <int P>
__global__ void ks_spread(StaticArgs s) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n) return;
  int b[3];
  double th[3][P], dth[3][P];
  ks_spline<P>(s, i, b, th, dth);
  const double *Hi = s.bx + 9;
  const int K[3] = {s.K1, s.K2, s.K3};
  double e[3];
  for (int ax = 0; ax < 3; ++ax) e[ax] = (s.d[3 * i] * Hi[ax] + s.d[3 * i + 1] * Hi[3 + ax] + s.d[3 * i + 2] * Hi[6 + ax]) * K[ax];
  double qi = s.with_q ? s.q[i] : 0.0;
  for (int j1 = 0; j1 < P; ++j1)
    for (int j2 = 0; j2 < P; ++j2)
      for (int j3 = 0; j3 < P; ++j3) {
        double v = (qi * th[0][j1] + e[0] * dth[0][j1]) * th[1][j2] * th[2][j3] + e[1] * th[0][j1] * dth[1][j2] * th[2][j3] +
                   e[2] * th[0][j1] * th[1][j2] * dth[2][j3];
        int i1 = (b[0] + j1) % s.K1, i2 = (b[1] + j2) % s.K2, i3 = (b[2] + j3) % s.K3;
        atomicAdd(&s.A[((size_t)i1 * s.K2 + i2) * s.K3 + i3].x, v);
      }
}

// One axis of an unnormalised complex 3D DFT, dst(m) = sum_k src(k) exp(sign 2 pi i m k / K).
__global__ void ks_dft(StaticArgs s, const double2 *src, double2 *dst, int axis, int sign) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int ng = s.K1 * s.K2 * s.K3;
  if (g >= ng) return;
  int k3 = g % s.K3, k2 = (g / s.K3) % s.K2, k1 = g / (s.K2 * s.K3);
  int K = axis == 0 ? s.K1 : axis == 1 ? s.K2 : s.K3;
  int m = axis == 0 ? k1 : axis == 1 ? k2 : k3;
  size_t stride = axis == 0 ? (size_t)s.K2 * s.K3 : axis == 1 ? (size_t)s.K3 : 1;
  size_t base = g - (size_t)m * stride;
  double re = 0, im = 0;
  for (int k = 0; k < K; ++k) {
    double sn, cs;
    sincospi(2.0 * sign * (double)((long long)m * k % K) / K, &sn, &cs);
    double2 v = src[base + k * stride];
    re += v.x * cs - v.y * sn;
    im += v.x * sn + v.y * cs;
  }
  dst[g] = make_double2(re, im);
}

template <int P>
__device__ double ks_modulus(int K, int m) {
  double th[P], dth[P];
  pgm::bspline<double, P, false>(0.0, th, dth, nullptr);
  double c = 0, sn = 0;
  for (int j = 0; j < P; ++j) {
    double a, b;
    sincospi(2.0 * (double)((long long)m * j % K) / K, &b, &a);
    c += th[j] * a;
    sn += th[j] * b;
  }
  return c * c + sn * sn;
}

// |b(m)|^-2 denominators with the patch of near-zero values (pme.py:106-131).
template <int P>
__device__ double ks_mod(int K, int m) {
  double v = ks_modulus<P>(K, m);
  if (v < 1e-7) v = 0.5 * (ks_modulus<P>(K, (m - 1 + K) % K) + ks_modulus<P>(K, (m + 1) % K));
  return v;
}

// Multiply by 2 G(m) over the full spectrum (pme.py:243-267, 370-376).
template <int P>
__global__ void ks_convolve(StaticArgs s, double2 *grid) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  int ng = s.K1 * s.K2 * s.K3;
  if (g >= ng) return;
  int k3 = g % s.K3, k2 = (g / s.K3) % s.K2, k1 = g / (s.K2 * s.K3);
  int m1 = k1 <= (s.K1 - 1) / 2 ? k1 : k1 - s.K1, m2 = k2 <= (s.K2 - 1) / 2 ? k2 : k2 - s.K2,
      m3 = k3 <= (s.K3 - 1) / 2 ? k3 : k3 - s.K3;
  if (s.K1 % 2 == 0 && k1 == s.K1 / 2) m1 = -s.K1 / 2;
  if (s.K2 % 2 == 0 && k2 == s.K2 / 2) m2 = -s.K2 / 2;
  if (s.K3 % 2 == 0 && k3 == s.K3 / 2) m3 = -s.K3 / 2;
  const double *Hi = s.bx + 9;
  double mv[3];
  for (int c = 0; c < 3; ++c) mv[c] = m1 * Hi[c * 3 + 0] + m2 * Hi[c * 3 + 1] + m3 * Hi[c * 3 + 2];
  double msq = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
  double G = 0;
  if (msq > 0) {
    G = exp(-pgm::PI * pgm::PI * msq / (s.beta * s.beta)) / (2.0 * pgm::PI * s.bx[18] * msq);
    G /= ks_mod<P>(s.K1, k1) * ks_mod<P>(s.K2, k2) * ks_mod<P>(s.K3, k3);
  }
  double2 v = grid[g];
  grid[g] = make_double2(2.0 * G * v.x, 2.0 * G * v.y);
}

// One warp per atom: row field over every other atom within the cutoff (the rows of
// forcefield.py:1140-1195 without their storage), the PME gather of phi = Re(grid), and the field
// -(rows + dU_rec/dd - c_self d) (forcefield.py:1428-1433).
template <int P>
__global__ void ks_field(StaticArgs s, const double2 *phi) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int i = warp;
  if (i >= s.n) return;
  const double *H = s.bx;
  double pix = s.pos[3 * i], piy = s.pos[3 * i + 1], piz = s.pos[3 * i + 2];
  double Ri = s.radius[i];
  double f[3] = {0, 0, 0};
  for (int j = lane; j < s.n; j += 32) {
    if (j == i) continue;
    double x = pix - s.pos[3 * j], y = piy - s.pos[3 * j + 1], z = piz - s.pos[3 * j + 2];
    pgm::min_image(x, y, z, H);
    double r2 = x * x + y * y + z * z;
    if (r2 >= s.cutoff * s.cutoff) continue;
    double r = sqrt(r2), Rk = s.radius[j];
    double a = 1.0 / sqrt(2.0 * (Ri * Ri + Rk * Rk));
    double A[4], B[4];
    pgm::erf_kernels<double>(a, r, A);
    pgm::erf_kernels<double>(s.beta, r, B);
    double G1 = A[1] - B[1], G2 = A[2] - B[2];
    double dk[3] = {s.d[3 * j], s.d[3 * j + 1], s.d[3 * j + 2]};
    double dkx = dk[0] * x + dk[1] * y + dk[2] * z;
    double c = -G2 * dkx - (s.with_q ? s.q[j] * G1 : 0.0);
    f[0] += c * x + G1 * dk[0];
    f[1] += c * y + G1 * dk[1];
    f[2] += c * z + G1 * dk[2];
  }
  int b[3];
  double th[3][P], dth[3][P];
  ks_spline<P>(s, i, b, th, dth);
  double g[3] = {0, 0, 0};
  for (int p = lane; p < P * P * P; p += 32) {
    int j1 = p / (P * P), j2 = (p / P) % P, j3 = p % P;
    int i1 = (b[0] + j1) % s.K1, i2 = (b[1] + j2) % s.K2, i3 = (b[2] + j3) % s.K3;
    double ph = phi[((size_t)i1 * s.K2 + i2) * s.K3 + i3].x;
    g[0] += ph * dth[0][j1] * th[1][j2] * th[2][j3];
    g[1] += ph * th[0][j1] * dth[1][j2] * th[2][j3];
    g[2] += ph * th[0][j1] * th[1][j2] * dth[2][j3];
  }
  for (int c = 0; c < 3; ++c) {
    f[c] = pgm::warp_sum<double>(f[c]);
    g[c] = pgm::warp_sum<double>(g[c]);
  }
  if (lane == 0) {
    const double *Hi = s.bx + 9;
    const int K[3] = {s.K1, s.K2, s.K3};
    if (s.bx[19] != 0.0) {  // a box the minimum image cannot serve: no value rather than a wrong one
      for (int bb = 0; bb < 3; ++bb) s.field[3 * i + bb] = nan("");
      return;
    }
    for (int bb = 0; bb < 3; ++bb) {
      double rec = g[0] * Hi[bb * 3 + 0] * K[0] + g[1] * Hi[bb * 3 + 1] * K[1] + g[2] * Hi[bb * 3 + 2] * K[2];
      s.field[3 * i + bb] = -(f[bb] + rec - s.c_self * s.d[3 * i + bb]);
    }
  }
}

// Every launch is checked as it is made, so an error is this call's own (a pending error of an
// earlier launch was refused on entry).
template <int P>
cudaError_t run_static(StaticArgs s, cudaStream_t st) {
  int ng = s.K1 * s.K2 * s.K3;
  int gb = (ng + 255) / 256;
  cudaError_t e;
#define PGM_STATIC_LAUNCH(...) \
  do {                         \
    __VA_ARGS__;               \
    e = cudaGetLastError();    \
    if (e != cudaSuccess) return e; \
  } while (0)
  PGM_STATIC_LAUNCH(ks_box_and_clear<<<gb, 256, 0, st>>>(s));
  PGM_STATIC_LAUNCH(ks_spread<P><<<(s.n + 127) / 128, 128, 0, st>>>(s));
  PGM_STATIC_LAUNCH(ks_dft<<<gb, 256, 0, st>>>(s, s.A, s.B, 2, -1));
  PGM_STATIC_LAUNCH(ks_dft<<<gb, 256, 0, st>>>(s, s.B, s.A, 1, -1));
  PGM_STATIC_LAUNCH(ks_dft<<<gb, 256, 0, st>>>(s, s.A, s.B, 0, -1));
  PGM_STATIC_LAUNCH(ks_convolve<P><<<gb, 256, 0, st>>>(s, s.B));
  PGM_STATIC_LAUNCH(ks_dft<<<gb, 256, 0, st>>>(s, s.B, s.A, 0, +1));
  PGM_STATIC_LAUNCH(ks_dft<<<gb, 256, 0, st>>>(s, s.A, s.B, 1, +1));
  PGM_STATIC_LAUNCH(ks_dft<<<gb, 256, 0, st>>>(s, s.B, s.A, 2, +1));
  PGM_STATIC_LAUNCH(ks_field<P><<<(s.n * 32 + 255) / 256, 256, 0, st>>>(s, s.A));
#undef PGM_STATIC_LAUNCH
  return cudaSuccess;
}

}  // namespace

extern "C" {

const char *pgm_static_last_error(void) { return g_static_err.c_str(); }

PgmStatus pgm_field_static(void *stream, int n_atoms, const double *pos, const double *box, const double *q,
                           const double *radius, double cutoff, double ewald_beta, const int *pme_grid, int pme_order,
                           int with_charges, const double *d, double *field) {
  if (!pos || !box || !radius || !d || !field || !pme_grid || (with_charges && !q))
    return serr(PGM_ERR_INVALID, "null argument");
  if (n_atoms <= 0 || n_atoms > PGM_STATIC_MAX_ATOMS)
    return serr(PGM_ERR_UNSUPPORTED, "pgm_field_static: n_atoms must be in 1.." + std::to_string(PGM_STATIC_MAX_ATOMS));
  const int K1 = pme_grid[0], K2 = pme_grid[1], K3 = pme_grid[2];
  if (K1 < pme_order || K2 < pme_order || K3 < pme_order || K1 > PGM_STATIC_MAX_K || K2 > PGM_STATIC_MAX_K ||
      K3 > PGM_STATIC_MAX_K || (long long)K1 * K2 * K3 > PGM_STATIC_MAX_GRID)
    return serr(PGM_ERR_UNSUPPORTED, "pgm_field_static: mesh sizes must be in order.." + std::to_string(PGM_STATIC_MAX_K) +
                                         " with at most " + std::to_string(PGM_STATIC_MAX_GRID) + " points");
  if (pme_order != 4 && pme_order != 6 && pme_order != 8) return serr(PGM_ERR_UNSUPPORTED, "pme_order must be 4, 6 or 8");
  if (!(cutoff > 0) || !(ewald_beta > 0)) return serr(PGM_ERR_INVALID, "cutoff and ewald_beta must be positive");
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)  // left by an earlier launch of the caller: not cleared here, not blamed on this call
    return serr(PGM_ERR_CUDA, std::string("pgm_field_static: an earlier CUDA error is pending: ") + cudaGetErrorString(e));
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return serr(PGM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return serr(PGM_ERR_UNSUPPORTED, "device index above 63");
  int sdev = dev;
  e = cudaStreamGetDevice((cudaStream_t)stream, &sdev);
  if (e != cudaSuccess) return serr(PGM_ERR_CUDA, std::string("cudaStreamGetDevice: ") + cudaGetErrorString(e));
  if (sdev != dev)  // the scratch address below belongs to the current device
    return serr(PGM_ERR_INVALID, "pgm_field_static: the stream belongs to device " + std::to_string(sdev) +
                                     ", the current device is " + std::to_string(dev));
  double *base = nullptr;
  {
    // set-up, once per device with that device current: the device address of the array
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_ptr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_field_scratch);
      if (e != cudaSuccess) return serr(PGM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_static_ptr[dev] = static_cast<double *>(p);
    }
    base = g_static_ptr[dev];
  }
  StaticArgs s;
  s.n = n_atoms; s.K1 = K1; s.K2 = K2; s.K3 = K3;
  s.cutoff = cutoff; s.beta = ewald_beta; s.c_self = 4.0 * ewald_beta * ewald_beta * ewald_beta / (3.0 * pgm::SQRT_PI);
  s.pos = pos; s.box = box; s.q = q; s.radius = radius; s.d = d; s.with_q = with_charges; s.field = field;
  s.A = reinterpret_cast<double2 *>(base);
  s.B = reinterpret_cast<double2 *>(base) + PGM_STATIC_MAX_GRID;
  s.bx = base + 4 * (size_t)PGM_STATIC_MAX_GRID;
  cudaStream_t st = (cudaStream_t)stream;
  e = pme_order == 4 ? run_static<4>(s, st) : pme_order == 6 ? run_static<6>(s, st) : run_static<8>(s, st);
  if (e != cudaSuccess) return serr(PGM_ERR_CUDA, std::string("pgm_field_static launch: ") + cudaGetErrorString(e));
  return PGM_OK;
}

}  // extern "C"
