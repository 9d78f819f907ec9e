// pgm_pimd.cu -- path-integral MD of flexible molecules on the GPU: the ring-polymer integrator
// around the batched force field (the beads of a ring polymer are the systems of one engine
// batch, so every bead's pair rows, PME and induced-dipole solve run in the same launches).
//
// The reference's PIMDIntegrator (pgm_jax/md/pimd.py:484-700, RingPolymer :183-296, PILEStep
// :358-440): BAOAB with the free ring polymer in normal modes,
//   B(dt/2)  p += dt/2 f                    (k_pimd_kick)
//   A(dt/2) O(dt) A(dt/2) in normal modes   (k_pimd_aoa: Cayley free step, PILE-L, Cayley step)
//   forces, B(dt/2).
// Normal modes q~_l = sum_j C_jl q_j (C real orthonormal: centroid, cos/sin pairs, alternating
// mode), omega_l = 2 omega_P sin(pi idx_l / P).  Cayley step of length h per mode:
//   p' = [(1 - x) p - m w^2 h q] / (1 + x),  q' = [h p / m + (1 - x) q] / (1 + x),  x = (w h / 2)^2.
// PILE-L: p <- c p + sqrt((1 - c^2) m P kB T) xi with c = exp(-gamma_l dt) per mode.
//
// Layout: q, p, f are the engine's batch arrays, bead-major: atom i of bead k at (k N + i).
// One warp per (atom, Cartesian component): lane k holds bead k (P <= 32), the transforms are
// warp shuffles.  The q-TIP4P/F intramolecular term of flexible water (quartic Morse O-H bonds and
// a harmonic bend, pgm_jax/models/water.py:33-69) is added to the forces by k_water_bonded.
#include <cuda_runtime.h>

#include <string>

#include "../../include/pgm_b200.h"

namespace {

thread_local std::string g_pimd_err;

#define PCK(call)                                                        \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      g_pimd_err = std::string(#call) + ": " + cudaGetErrorString(e_);   \
      return PGM_ERR_CUDA;                                               \
    }                                                                    \
  } while (0)

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// One standard normal per (seed, step, stream index) (splitmix64 hash, Box-Muller).
__device__ __forceinline__ double normal01(unsigned long long seed, unsigned long long step, unsigned long long idx) {
  unsigned long long h = mix64(seed ^ mix64(step * 0x100000001B3ull + idx));
  unsigned long long h2 = mix64(h ^ 0xD1B54A32D192ED03ull);
  double u1 = ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  double u2 = ((h2 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

__global__ void k_pimd_kick(long long n3, double h, const double *f, double *p) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n3) p[t] += h * f[t];
}

// The Cayley free ring-polymer step of length h for mode frequency w and mass m.
__device__ __forceinline__ void cayley(double w, double m, double h, double &q, double &p) {
  const double x = 0.25 * w * w * h * h, den = 1.0 / (1.0 + x);
  const double pn = ((1.0 - x) * p - m * w * w * h * q) * den;
  const double qn = (h * p / m + (1.0 - x) * q) * den;
  q = qn;
  p = pn;
}

struct PimdArgs {
  int P, N;
  const double *C;      // (P, P) row-major: C[j * P + l]
  const double *omega;  // (P,) rad/ps
  const double *gamma;  // (P,) 1/ps (all zero: RPMD)
  const double *mass;   // (N,) amu
  double dt, kTP;
  unsigned long long seed;
  unsigned long long *counter;
  const double *cscale;  // PILE-G: the centroid's Bussi factor (null: none)
};

// One uniform in (0, 1) per (seed, step, stream index) (the hash of normal01).
__device__ __forceinline__ double uniform01(unsigned long long seed, unsigned long long step, unsigned long long idx) {
  unsigned long long h = mix64(seed ^ mix64(step * 0x100000001B3ull + idx));
  return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// Stream indices of the Bussi draws, above those of the per-(atom, component, mode) Langevin noise.
constexpr unsigned long long BUSSI_STREAM = 1ull << 48;

// PILE-G, step 1: the centroid kinetic energy K = sum_i,c p~0(i, c)^2 / (2 m_i) of the ring
// polymer, p~0 = sum_j C[j][0] p_j (one thread per atom component, block sums, one atomic each).
__global__ void k_centroid_ke(int P, int N, const double *C, const double *mass, const double *p, double *K) {
  __shared__ double red[8];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (t < 3LL * N) {
    const int i = (int)(t / 3);
    double p0 = 0.0;
    for (int j = 0; j < P; ++j) p0 += C[j * P] * p[(size_t)j * 3 * N + t];
    e = 0.5 * p0 * p0 / mass[i];
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w];
    atomicAdd(K, v);
  }
}

// PILE-G, step 2 (one thread): Bussi's exact rescaling factor (thermostats.py:279-335) for an O
// step of length h with time constant tau, from K = work[0] at kT with N_f = dof:
//   alpha^2 = c + (1 - c) f (R1^2 + S) + 2 R1 sqrt(c (1 - c) f),  f = K0 / (N_f K) = kT / (2 K),
// c = exp(-h / tau), R1 ~ N(0, 1), S ~ chi^2(N_f - 1) = 2 Gamma((N_f - 1) / 2), alpha with the
// sign of R1 + sqrt(c / ((1 - c) f)).  The Gamma variate by Marsaglia and Tsang's method (ACM TOMS
// 26, 363 (2000)), shape k = (N_f - 1) / 2 >= 1, at most 64 proposals (then its mode).
// work: [K, alpha, R1, S].
__global__ void k_bussi(double dof, double kT, double h, double tau, unsigned long long seed, const unsigned long long *counter,
                        double *work) {
  const unsigned long long step = *counter;
  const double K = fmax(work[0], 1e-30);
  const double c = exp(-h / tau), f = kT / (2.0 * K);
  const double r1 = normal01(seed, step, BUSSI_STREAM);
  const double k = 0.5 * (dof - 1.0), d = k - 1.0 / 3.0, cc = 1.0 / sqrt(9.0 * d);
  double g = d;
  for (int it = 0; it < 64; ++it) {
    const double x = normal01(seed, step, BUSSI_STREAM + 1 + 2 * it);
    double v = 1.0 + cc * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    const double u = uniform01(seed, step, BUSSI_STREAM + 2 + 2 * it);
    if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) {
      g = d * v;
      break;
    }
  }
  const double S = 2.0 * g;
  const double a2 = c + (1.0 - c) * f * (r1 * r1 + S) + 2.0 * r1 * sqrt(c * (1.0 - c) * f);
  const double sg = (r1 + sqrt(c / ((1.0 - c) * f))) < 0.0 ? -1.0 : 1.0;
  work[1] = sg * sqrt(fmax(a2, 0.0));
  work[2] = r1;
  work[3] = S;
}

__global__ void __launch_bounds__(256) k_pimd_aoa(PimdArgs A, double *q, double *p) {
  const int lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // (atom, component)
  if (w >= 3LL * A.N) return;
  const int i = (int)(w / 3), c = (int)(w % 3);
  const int P = A.P;
  const bool on = lane < P;
  const size_t off = (size_t)i * 3 + c, stride = (size_t)A.N * 3;
  double qb = on ? q[(size_t)lane * stride + off] : 0.0, pb = on ? p[(size_t)lane * stride + off] : 0.0;
  // to normal modes: lane l <- sum_j C[j][l] x_j
  double qn = 0.0, pn = 0.0;
  for (int j = 0; j < P; ++j) {
    double cj = on ? A.C[j * P + lane] : 0.0;
    qn += cj * __shfl_sync(0xffffffffu, qb, j);
    pn += cj * __shfl_sync(0xffffffffu, pb, j);
  }
  if (on) {
    const double m = A.mass[i], wl = A.omega[lane], h = 0.5 * A.dt;
    cayley(wl, m, h, qn, pn);
    const double g = A.gamma[lane];
    if (lane == 0 && A.cscale) {
      pn *= *A.cscale;  // PILE-G: the centroid rescaled by Bussi's factor
    } else if (g > 0.0) {
      const double cc = exp(-g * A.dt);
      const unsigned long long step = *A.counter;
      const double xi = normal01(A.seed, step, ((unsigned long long)off * 32ull + lane));
      pn = cc * pn + sqrt((1.0 - cc * cc) * m * A.kTP) * xi;
    }
    cayley(wl, m, h, qn, pn);
  }
  // back to beads: lane j <- sum_l C[j][l] y_l
  double qo = 0.0, po = 0.0;
  for (int l = 0; l < P; ++l) {
    double cl = on ? A.C[lane * P + l] : 0.0;
    qo += cl * __shfl_sync(0xffffffffu, qn, l);
    po += cl * __shfl_sync(0xffffffffu, pn, l);
  }
  if (on) {
    q[(size_t)lane * stride + off] = qo;
    p[(size_t)lane * stride + off] = po;
  }
}

__global__ void k_pimd_count(unsigned long long *counter) { *counter += 1; }

// q-TIP4P/F water (O, H, H consecutive from `first`): D [x^2 - x^3 + 7/12 x^4], x = alpha (r - r0)
// per O-H bond, k_theta (theta - theta0)^2 / 2; forces added to f, energy per system.
__global__ void k_water_bonded(int nmol, const int *first, const int *msys, const double *x, double D, double alpha, double r0,
                               double kth, double th0, double *f, double *energy) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nmol) return;
  const int o = first[m], h1 = o + 1, h2 = o + 2;
  double u[3], v[3];
  for (int k = 0; k < 3; ++k) {
    u[k] = x[3 * h1 + k] - x[3 * o + k];
    v[k] = x[3 * h2 + k] - x[3 * o + k];
  }
  const double r1 = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]), r2 = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double e = 0.0, g1, g2;
  {
    double a = alpha * (r1 - r0);
    e += D * (a * a - a * a * a + 7.0 / 12.0 * a * a * a * a);
    g1 = D * alpha * (2.0 * a - 3.0 * a * a + 7.0 / 3.0 * a * a * a);  // dE/dr1
    a = alpha * (r2 - r0);
    e += D * (a * a - a * a * a + 7.0 / 12.0 * a * a * a * a);
    g2 = D * alpha * (2.0 * a - 3.0 * a * a + 7.0 / 3.0 * a * a * a);
  }
  const double uv = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
  double cs = uv / (r1 * r2);
  cs = fmin(1.0, fmax(-1.0, cs));
  const double th = acos(cs), sn = fmax(sqrt(1.0 - cs * cs), 1e-12);
  e += 0.5 * kth * (th - th0) * (th - th0);
  const double dEdth = kth * (th - th0);
  // d theta / du = -(v / (r1 r2) - cs u / r1^2) / sin(theta), likewise for v
  double fu[3], fv[3];
  for (int k = 0; k < 3; ++k) {
    const double dthu = -(v[k] / (r1 * r2) - cs * u[k] / (r1 * r1)) / sn;
    const double dthv = -(u[k] / (r1 * r2) - cs * v[k] / (r2 * r2)) / sn;
    fu[k] = -(g1 * u[k] / r1 + dEdth * dthu);  // force on H1 (u = H1 - O)
    fv[k] = -(g2 * v[k] / r2 + dEdth * dthv);
  }
  for (int k = 0; k < 3; ++k) {
    f[3 * h1 + k] += fu[k];
    f[3 * h2 + k] += fv[k];
    f[3 * o + k] -= fu[k] + fv[k];
  }
  if (energy) atomicAdd(&energy[msys[m]], e);
}

}  // namespace

extern "C" {

PgmStatus pgm_pimd_kick(void *stream, long long n3, double h, const double *forces, double *mom) {
  if (!forces || !mom || n3 < 0) return PGM_ERR_INVALID;
  if (n3 == 0) return PGM_OK;
  k_pimd_kick<<<(unsigned)((n3 + 255) / 256), 256, 0, (cudaStream_t)stream>>>(n3, h, forces, mom);
  PCK(cudaGetLastError());
  return PGM_OK;
}

PgmStatus pgm_pimd_free_thermostat(void *stream, int beads, int n_atoms, const double *C, const double *omega, const double *gamma,
                                   const double *mass, double dt, double kT_P, uint64_t seed, uint64_t *counter, double *pos,
                                   double *mom) {
  return pgm_pimd_free_thermostat_scaled(stream, beads, n_atoms, C, omega, gamma, mass, dt, kT_P, seed, counter, pos, mom, nullptr);
}

PgmStatus pgm_pimd_centroid_bussi(void *stream, int beads, int n_atoms, const double *C, const double *mass, double dt, double kT_P,
                                  double tau, uint64_t seed, const uint64_t *counter, const double *mom, double *work) {
  if (beads < 1 || beads > 32 || n_atoms < 1 || !C || !mass || !counter || !mom || !work || !(tau > 0.0) || !(dt > 0.0))
    return PGM_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  PCK(cudaMemsetAsync(work, 0, sizeof(double), st));
  const long long n3 = 3LL * n_atoms;
  k_centroid_ke<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(beads, n_atoms, C, mass, mom, work);
  PCK(cudaGetLastError());
  k_bussi<<<1, 1, 0, st>>>(3.0 * n_atoms, kT_P, dt, tau, seed, reinterpret_cast<const unsigned long long *>(counter), work);
  PCK(cudaGetLastError());
  return PGM_OK;
}

PgmStatus pgm_pimd_free_thermostat_scaled(void *stream, int beads, int n_atoms, const double *C, const double *omega,
                                          const double *gamma, const double *mass, double dt, double kT_P, uint64_t seed,
                                          uint64_t *counter, double *pos, double *mom, const double *centroid_scale) {
  if (beads < 1 || beads > 32 || n_atoms < 0 || !C || !omega || !gamma || !mass || !counter || !pos || !mom)
    return PGM_ERR_INVALID;
  if (n_atoms == 0) return PGM_OK;
  PimdArgs A{beads, n_atoms, C, omega, gamma, mass, dt, kT_P, seed, reinterpret_cast<unsigned long long *>(counter),
             centroid_scale};
  const long long warps = 3LL * n_atoms;
  k_pimd_aoa<<<(unsigned)((warps + 7) / 8), 256, 0, (cudaStream_t)stream>>>(A, pos, mom);
  PCK(cudaGetLastError());
  k_pimd_count<<<1, 1, 0, (cudaStream_t)stream>>>(reinterpret_cast<unsigned long long *>(counter));
  PCK(cudaGetLastError());
  return PGM_OK;
}

PgmStatus pgm_water_bonded(void *stream, int n_mol, const int32_t *first_atom, const int32_t *mol_system, const double *pos,
                           const double *params, double *forces, double *energy) {
  if (n_mol < 0 || !first_atom || !mol_system || !pos || !params || !forces) return PGM_ERR_INVALID;
  if (n_mol == 0) return PGM_OK;
  k_water_bonded<<<(n_mol + 127) / 128, 128, 0, (cudaStream_t)stream>>>(n_mol, first_atom, mol_system, pos, params[0], params[1],
                                                                        params[2], params[3], params[4], forces, energy);
  PCK(cudaGetLastError());
  return PGM_OK;
}

const char *pgm_pimd_last_error(void) { return g_pimd_err.c_str(); }

}  // extern "C"
