// pgm_md.cu -- rigid-molecule MD driver on the GPU: the caller of the force field in the MD
// benchmarks (the role of pgm_jax/md/integrate.py:743-761 with md/rigid.py and the Langevin
// O-step of md/thermostats.py:195-240).
//
// Rigid bodies: centre of mass X, orientation quaternion q (body -> space), COM momentum P and
// body-frame angular momentum L; atoms at X + R(q) b_i with b_i in the principal frame.  With
// Langevin friction (gamma > 0) one step is B A O A (forces) B; in NVE (gamma = 0) it is B A
// (forces) B with one drift of the full step, as integrate.py:743-761.  B: half kicks of P and L
// (torque rotated into the body frame).  A: the drift of X and the free rotor by exact rotations
// about the principal axes 3, 2, 1, 2, 3 (half, half, full, half, half) -- the splitting of
// Dullweber, Leimkuhler and McLachlan (J. Chem. Phys. 107, 5840 (1997)), in quaternion form the
// NO_SQUISH integrator of Miller et al. (J. Chem. Phys. 116, 8649 (2002)) that the reference runs.
// O: P <- c P + sqrt((1 - c^2) M kT) xi, L_k <- c L_k + sqrt((1 - c^2) I_k kT) xi with
// c = exp(-gamma dt).  One thread per molecule; FP64 throughout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pgm_b200.h"

namespace {

struct MDDev {
  int nmol;
  const int *mol_start;
  const double *mass;     // (N)
  const double *body;     // (N, 3) principal-frame coordinates
  const double *inertia;  // (M, 3)
  const double *mtot;     // (M)
  const int *msys;        // (M) system of every molecule
};

__device__ __forceinline__ void quat_rot(const double *q, double R[9]) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y - w * z);     R[2] = 2 * (x * z + w * y);
  R[3] = 2 * (x * y + w * z);     R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z - w * x);
  R[6] = 2 * (x * z - w * y);     R[7] = 2 * (y * z + w * x);     R[8] = 1 - 2 * (x * x + y * y);
}

// Free rotation about body axis k for time t: L rotates by -phi about e_k, q <- q (x) exp(phi/2 e_k).
__device__ __forceinline__ void rotate_axis(int k, double t, const double *I, double *L, double *q) {
  double phi = t * L[k] / I[k];
  double sh, ch;
  sincos(0.5 * phi, &sh, &ch);
  const double c = 1.0 - 2.0 * sh * sh, s = 2.0 * sh * ch;  // cos phi, sin phi by the double-angle identities
  int a = (k + 1) % 3, b = (k + 2) % 3;
  double La = L[a], Lb = L[b];
  L[a] = c * La + s * Lb;
  L[b] = -s * La + c * Lb;
  double e[3] = {0, 0, 0};
  e[k] = sh;
  double w = q[0], x = q[1], y = q[2], z = q[3];
  // q (x) (ch, e)
  double nw = w * ch - x * e[0] - y * e[1] - z * e[2];
  double nx = w * e[0] + x * ch + y * e[2] - z * e[1];
  double ny = w * e[1] - x * e[2] + y * ch + z * e[0];
  double nz = w * e[2] + x * e[1] - y * e[0] + z * ch;
  double n = rsqrt(nw * nw + nx * nx + ny * ny + nz * nz);
  q[0] = nw * n; q[1] = nx * n; q[2] = ny * n; q[3] = nz * n;
}

__device__ __forceinline__ void free_rotor(double h, const double *I, double *L, double *q) {
  rotate_axis(2, 0.5 * h, I, L, q);
  rotate_axis(1, 0.5 * h, I, L, q);
  rotate_axis(0, h, I, L, q);
  rotate_axis(1, 0.5 * h, I, L, q);
  rotate_axis(2, 0.5 * h, I, L, q);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Two standard normals from a counter (splitmix64 hash, Box-Muller).
__device__ __forceinline__ void normals(unsigned long long seed, unsigned long long step, int mol, int k, double &g0, double &g1) {
  unsigned long long h = mix64(seed ^ mix64(step * 0x100000001B3ull + (unsigned long long)mol * 8 + k));
  unsigned long long h2 = mix64(h);
  double u1 = ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  double u2 = ((h2 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  double r = sqrt(-2.0 * log(u1)), sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  g0 = r * cs;
  g1 = r * sn;
}

// Half kick of P and L from the atom forces.
__device__ __forceinline__ void half_kick(const MDDev &d, int m, double dt, const double *F, const double *R, double *P,
                                          double *L) {
  double f[3] = {0, 0, 0}, tau[3] = {0, 0, 0};
  for (int i = d.mol_start[m]; i < d.mol_start[m + 1]; ++i) {
    const double *b = d.body + 3 * i;
    double r[3] = {R[0] * b[0] + R[1] * b[1] + R[2] * b[2], R[3] * b[0] + R[4] * b[1] + R[5] * b[2],
                   R[6] * b[0] + R[7] * b[1] + R[8] * b[2]};
    const double *fi = F + 3 * i;
    f[0] += fi[0]; f[1] += fi[1]; f[2] += fi[2];
    tau[0] += r[1] * fi[2] - r[2] * fi[1];
    tau[1] += r[2] * fi[0] - r[0] * fi[2];
    tau[2] += r[0] * fi[1] - r[1] * fi[0];
  }
  for (int c = 0; c < 3; ++c) P[c] += 0.5 * dt * f[c];
  // body frame: R^T tau
  for (int c = 0; c < 3; ++c) L[c] += 0.5 * dt * (R[0 * 3 + c] * tau[0] + R[1 * 3 + c] * tau[1] + R[2 * 3 + c] * tau[2]);
}

__global__ void k_md_begin(MDDev d, double dt, double gamma, const double *kT, unsigned long long seed,
                           const unsigned long long *counter, const double *F, double *X, double *Q, double *P, double *L,
                           double *pos, const double *box) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a programmatic dependent: the forces are complete
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= d.nmol) return;
  unsigned long long step = *counter;
  double x[3] = {X[3 * m], X[3 * m + 1], X[3 * m + 2]}, q[4] = {Q[4 * m], Q[4 * m + 1], Q[4 * m + 2], Q[4 * m + 3]};
  double p[3] = {P[3 * m], P[3 * m + 1], P[3 * m + 2]}, l[3] = {L[3 * m], L[3 * m + 1], L[3 * m + 2]};
  const double *I = d.inertia + 3 * m;
  double M = d.mtot[m];
  double R[9];
  quat_rot(q, R);
  if (F) half_kick(d, m, dt, F, R, p, l);
  if (gamma > 0) {  // A(dt/2) O A(dt/2)
    for (int c = 0; c < 3; ++c) x[c] += 0.5 * dt * p[c] / M;
    free_rotor(0.5 * dt, I, l, q);
    double c = exp(-gamma * dt), t = kT[d.msys[m]];
    double g[6];
    normals(seed, step, m, 0, g[0], g[1]);
    normals(seed, step, m, 1, g[2], g[3]);
    normals(seed, step, m, 2, g[4], g[5]);
    double sp = sqrt((1 - c * c) * M * t);
    for (int k = 0; k < 3; ++k) p[k] = c * p[k] + sp * g[k];
    for (int k = 0; k < 3; ++k) l[k] = c * l[k] + sqrt((1 - c * c) * I[k] * t) * g[3 + k];
    for (int c = 0; c < 3; ++c) x[c] += 0.5 * dt * p[c] / M;
    free_rotor(0.5 * dt, I, l, q);
  } else {  // NVE: A(dt)
    for (int c = 0; c < 3; ++c) x[c] += dt * p[c] / M;
    free_rotor(dt, I, l, q);
  }
  // keep the centre of mass in the box (sequential reduction by the lattice vectors)
  const double *H = box + 9 * d.msys[m];
  for (int c = 2; c >= 0; --c) {
    double u = x[c] / H[c * 3 + c];
    double n = floor(u);
    if (n != 0.0)
      for (int j = 0; j <= c; ++j) x[j] -= n * H[c * 3 + j];
  }
  quat_rot(q, R);
  for (int i = d.mol_start[m]; i < d.mol_start[m + 1]; ++i) {
    const double *b = d.body + 3 * i;
    pos[3 * i] = x[0] + R[0] * b[0] + R[1] * b[1] + R[2] * b[2];
    pos[3 * i + 1] = x[1] + R[3] * b[0] + R[4] * b[1] + R[5] * b[2];
    pos[3 * i + 2] = x[2] + R[6] * b[0] + R[7] * b[1] + R[8] * b[2];
  }
  for (int c = 0; c < 3; ++c) { X[3 * m + c] = x[c]; P[3 * m + c] = p[c]; L[3 * m + c] = l[c]; }
  for (int c = 0; c < 4; ++c) Q[4 * m + c] = q[c];
}

__global__ void k_md_end(MDDev d, double dt, const double *F, const double *Q, double *P, double *L,
                         unsigned long long *counter) {
  asm volatile("griddepcontrol.wait;" ::: "memory");  // a programmatic dependent: the forces are complete
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0) *counter += 1;  // the Langevin noise counter of the next step
  if (m >= d.nmol) return;
  double q[4] = {Q[4 * m], Q[4 * m + 1], Q[4 * m + 2], Q[4 * m + 3]};
  double p[3] = {P[3 * m], P[3 * m + 1], P[3 * m + 2]}, l[3] = {L[3 * m], L[3 * m + 1], L[3 * m + 2]};
  double R[9];
  quat_rot(q, R);
  half_kick(d, m, dt, F, R, p, l);
  for (int c = 0; c < 3; ++c) { P[3 * m + c] = p[c]; L[3 * m + c] = l[c]; }
}

// Kinetic energy per system: sum P^2 / 2M + sum L_k^2 / 2 I_k.
__global__ void k_md_kinetic(MDDev d, const double *P, const double *L, double *ke) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= d.nmol) return;
  double M = d.mtot[m];
  const double *I = d.inertia + 3 * m;
  double e = 0;
  for (int c = 0; c < 3; ++c) e += P[3 * m + c] * P[3 * m + c] / (2 * M) + L[3 * m + c] * L[3 * m + c] / (2 * I[c]);
  atomicAdd(&ke[d.msys[m]], e);
}

// Momenta (linear and angular) of every molecule times the factor of its system (replica
// exchange: sqrt(T_new / T_old) for a configuration that changes temperature, remd.py:571-611).
__global__ void k_md_scale(MDDev d, const double *factor, double *P, double *L) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= d.nmol) return;
  double f = factor[d.msys[m]];
  for (int c = 0; c < 3; ++c) {
    P[3 * m + c] *= f;
    L[3 * m + c] *= f;
  }
}

thread_local std::string g_md_err;

}  // namespace

struct PgmRigid {
  int device = 0, nmol = 0, nsys = 0;
  int *mol_start = nullptr, *msys = nullptr;
  double *mass = nullptr, *body = nullptr, *inertia = nullptr, *mtot = nullptr;
  unsigned long long *counter = nullptr;
  MDDev dev() const { return MDDev{nmol, mol_start, mass, body, inertia, mtot, msys}; }
};

#define MDCK(call)                                                  \
  do {                                                              \
    cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) {                                        \
      g_md_err = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return PGM_ERR_CUDA;                                          \
    }                                                               \
  } while (0)

// A launch with programmatic stream serialization: the kernel may be scheduled while its
// predecessor drains and waits (griddepcontrol.wait) for its completion before touching data.
template <typename... KArgs, typename... Args>
static cudaError_t launch_dependent(void (*k)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, args...);
}

extern "C" {

const char *pgm_rigid_last_error(void) { return g_md_err.c_str(); }

PgmStatus pgm_rigid_create(int n_mol, const int32_t *mol_start, const int32_t *mol_system, const double *masses,
                           const double *body, const double *inertia, int device, PgmRigid **out) {
  if (n_mol <= 0 || !mol_start || !mol_system || !masses || !body || !inertia || !out) return PGM_ERR_INVALID;
  int n = mol_start[n_mol];
  std::vector<double> mt(n_mol, 0.0);
  int nsys = 0;
  for (int m = 0; m < n_mol; ++m) {
    if (mol_start[m + 1] <= mol_start[m]) return PGM_ERR_INVALID;
    for (int i = mol_start[m]; i < mol_start[m + 1]; ++i) mt[m] += masses[i];
    for (int k = 0; k < 3; ++k)
      if (!(inertia[3 * m + k] > 0)) return PGM_ERR_UNSUPPORTED;  // linear or single-atom bodies
    nsys = std::max(nsys, mol_system[m] + 1);
  }
  MDCK(cudaSetDevice(device));
  PgmRigid *r = new PgmRigid();
  r->device = device;
  r->nmol = n_mol;
  r->nsys = nsys;
  auto up = [&](auto **dst, const auto *src, size_t cnt) -> cudaError_t {
    cudaError_t e = cudaMalloc((void **)dst, sizeof(**dst) * cnt);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, src, sizeof(**dst) * cnt, cudaMemcpyHostToDevice);
  };
  MDCK(up(&r->mol_start, mol_start, n_mol + 1));
  MDCK(up(&r->msys, mol_system, n_mol));
  MDCK(up(&r->mass, masses, n));
  MDCK(up(&r->body, body, 3 * (size_t)n));
  MDCK(up(&r->inertia, inertia, 3 * (size_t)n_mol));
  MDCK(up(&r->mtot, mt.data(), n_mol));
  MDCK(cudaMalloc(&r->counter, sizeof(unsigned long long)));
  MDCK(cudaMemset(r->counter, 0, sizeof(unsigned long long)));
  *out = r;
  return PGM_OK;
}

PgmStatus pgm_rigid_destroy(PgmRigid *r) {
  if (!r) return PGM_ERR_INVALID;
  cudaSetDevice(r->device);
  cudaFree(r->mol_start); cudaFree(r->msys); cudaFree(r->mass); cudaFree(r->body); cudaFree(r->inertia); cudaFree(r->mtot); cudaFree(r->counter);
  delete r;
  return PGM_OK;
}

PgmStatus pgm_rigid_set_step(PgmRigid *r, uint64_t step) {
  if (!r) return PGM_ERR_INVALID;
  unsigned long long v = step;
  MDCK(cudaMemcpy(r->counter, &v, sizeof(v), cudaMemcpyHostToDevice));
  return PGM_OK;
}

PgmStatus pgm_rigid_begin_step(PgmRigid *r, void *stream, double dt, double gamma, const double *kT, uint64_t seed,
                               const double *forces, double *com, double *quat, double *mom, double *angmom, double *pos,
                               const double *box) {
  if (!r || !com || !quat || !mom || !angmom || !pos || !box || (gamma > 0 && !kT)) return PGM_ERR_INVALID;
  MDCK(launch_dependent(k_md_begin, (r->nmol + 127) / 128, 128, (cudaStream_t)stream, r->dev(), dt, gamma, kT, seed,
                        (const unsigned long long *)r->counter, forces, com, quat, mom, angmom, pos, box));
  return PGM_OK;
}

PgmStatus pgm_rigid_end_step(PgmRigid *r, void *stream, double dt, const double *forces, const double *quat, double *mom,
                             double *angmom) {
  if (!r || !forces || !quat || !mom || !angmom) return PGM_ERR_INVALID;
  MDCK(launch_dependent(k_md_end, (r->nmol + 127) / 128, 128, (cudaStream_t)stream, r->dev(), dt, forces, quat, mom, angmom,
                        r->counter));
  return PGM_OK;
}

PgmStatus pgm_rigid_kinetic(PgmRigid *r, void *stream, const double *mom, const double *angmom, double *ke) {
  if (!r || !mom || !angmom || !ke) return PGM_ERR_INVALID;
  MDCK(cudaMemsetAsync(ke, 0, sizeof(double) * r->nsys, (cudaStream_t)stream));
  k_md_kinetic<<<(r->nmol + 127) / 128, 128, 0, (cudaStream_t)stream>>>(r->dev(), mom, angmom, ke);
  MDCK(cudaGetLastError());
  return PGM_OK;
}

PgmStatus pgm_rigid_scale_momenta(PgmRigid *r, void *stream, const double *factor, double *mom, double *angmom) {
  if (!r || !factor || !mom || !angmom) return PGM_ERR_INVALID;
  k_md_scale<<<(r->nmol + 127) / 128, 128, 0, (cudaStream_t)stream>>>(r->dev(), factor, mom, angmom);
  MDCK(cudaGetLastError());
  return PGM_OK;
}

// Graph helpers for callers without a CUDA binding of their own: capture a sequence of engine
// calls on `stream` into an executable graph and replay it.
PgmStatus pgm_graph_begin(void *stream) {
  MDCK(cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeRelaxed));
  return PGM_OK;
}

PgmStatus pgm_graph_end(void *stream, void **exec_out) {
  if (!exec_out) return PGM_ERR_INVALID;
  cudaGraph_t g;
  MDCK(cudaStreamEndCapture((cudaStream_t)stream, &g));
  cudaGraphExec_t ex;
  MDCK(cudaGraphInstantiateWithFlags(&ex, g, cudaGraphInstantiateFlagUseNodePriority));  // kernels keep their launch priority
  MDCK(cudaGraphDestroy(g));
  *exec_out = (void *)ex;
  return PGM_OK;
}

PgmStatus pgm_graph_launch(void *exec, void *stream) {
  if (!exec) return PGM_ERR_INVALID;
  MDCK(cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream));
  return PGM_OK;
}

PgmStatus pgm_graph_destroy(void *exec) {
  if (!exec) return PGM_ERR_INVALID;
  MDCK(cudaGraphExecDestroy((cudaGraphExec_t)exec));
  return PGM_OK;
}

}  // extern "C"
