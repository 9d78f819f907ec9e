// pgm_kernels.cuh -- the sm_100a kernels of the pGM step.
//
// Layout in HBM (all systems of a batch concatenated; a block never straddles two systems):
//   atoms      SoA per-atom parameters (T) and state; 3-vectors as 16/32-byte v4<T> for single loads
//   rows       [atom][capacity] structure of arrays: partner k (int32), x, y, z, G0..G3 (T);
//              molecule partners first (the rigid special table), then the in-cutoff neighbours
//   PME        per system a real grid K1 x K2 x K3 (k3 fastest) and a half-complex grid
//              K1 x K2 x (K3/2 + 1), both as flat offsets into batch-wide buffers
//   reductions per-system FP64 accumulators (CGSys, EnergyAcc), filled by block partials + atomics
//
// Reference correspondence (pgm_jax/md/...): row build forcefield.py:1140-1195, radial kernels
// kernels.py:76-118 + forcefield.py:1318-1338, direct field forcefield.py:1395-1433, PME
// pme.py:243-411, CG forcefield.py:1714-1821, start forcefield.py:1917-2008, energy and forces
// forcefield.py:2011-2045,2294-2430, strain derivative forcefield.py:608-662,2628-2695.
#pragma once
#include "pgm_device.cuh"
#include "pgm_nn.cuh"

namespace pgm {

template <typename T>
struct Dev {
  int nsys, nt, nmol, mc, ncell, ncov;
  int order;
  int induce, perm, lj, lj_lrc;
  double beta, cutoff, c_self, tol, peek;
  double skin;            // Verlet skin of the candidate list
  int cc;                 // candidate capacity per atom
  int *nb_flag;           // candidate list must be rebuilt
  long long *nb_builds;   // rebuild counter
  int *cand, *ncand;      // candidates (N, cc) and counts
  double4 *pos_ref;       // positions at the last rebuild
  double4 *pos4;          // positions this step, .w = molecule
  float4 *pos4f;          // FP32 rows (mixed precision): the positions wrapped into the box, .w = molecule
  int max_iter;
  const SysInfo *sys;
  BoxInfo *box;
  CGSys *cg;
  EnergyAcc *eacc;
  unsigned *status;
  // block maps (warp-per-atom and thread-per-atom kernels)
  const int *wb_sys, *wb_atom0, *tb_sys, *tb_atom0;
  // atoms
  const int *sysid, *molid, *molfirst, *molend, *mol_start;
  const T *q, *radius, *alpha, *ialpha, *rminh, *seps;
  const v4<T> *qls;  // per atom (q, R*/2, sqrt(eps), 0): one load per partner in the force pass
  const double *mass;
  const int *cov_start, *cov_j, *cov_i_flat, *cov_j_flat;
  const double *cov_c, *cov_c_flat;
  // per step
  const double *pos;
  int4 *base;
  v4<T> *frac;
  double4 *pperm, *off;
  int *cell_of, *slot_of, *cell_count, *cell_start, *cell_atoms;
  double4 *spos;  // positions in cell order, .w = molecule
  const int *idx;
  int idx_width;
  // rows
  int *rn, *rnsp, *rk;
  T *rx, *ry, *rz, *rg0, *rg1, *rg2, *rg3;
  int *max_count;  // [0] largest electrostatic (or only) part, [1] largest van der Waals part
  // split rows: the electrostatic part of a row is [0, mce), the van der Waals part [mce, mc) with
  // its counts in rnv (null: one cutoff, mce == mc); rce2 = elec_cutoff^2
  int mce;
  int *rnv;
  double rce2;
  // the learned guess's graph (the row entries with float(r^2) < nn_rg2): per atom up to nn_emax
  // edges (x, y, z, partner bits) in row order and the full count, written by the row build when
  // nn_e4 is set (the consumers read the first nn_emax), with the pair kernels G1, G2 of each edge
  // in nn_g (same slots)
  float4 *nn_e4;
  float2 *nn_g;
  int *nn_ne;
  int nn_emax;
  float nn_rg2;
  // local preconditioner (local_niter > 0, forcefield.py:1766-1792): the row entries with
  // r^2 < lc2, entry-major (entry e of atom i at e nt + i, at most sh_max, sh_n per atom): partner
  // displacement, G1 and G2 written by the row build; the inner CG's vectors
  // rr (LRR), alpha rr (LZZ), its directions (LP0 / LP1, alternating), and r_new - r_old of the
  // outer update (DR)
  int *sh_n;
  int sh_max;
  double lc2;
  int *c_k;
  T *c_x, *c_y, *c_z, *c_g1, *c_g2;
  v4<T> *LRR, *LZZ, *LP0, *LP1, *DR;
  // iEL/0-SCF shadow energy: delta (Dl) and the reciprocal potential of delta alone (Phi2);
  // iel_keep = 1 - 1/omega for pairs inside a preconditioner block when iel_keep_on
  const v4<T> *Dl;
  const T *Phi2;
  double iel_keep;
  int iel_keep_on;
  // vectors
  v4<T> *X, *R, *Z, *P, *AP, *B, *D;
  v4<T> *F;  // row field of a sweep (computed concurrently with the PME chain)
  v4<T> *Fp; // the early-fork schedule: row field of the previous CG direction
  // grids
  T *Q, *Phi, *Ginf;
  c2<T> *C;
  const c2<T> *tw;
  const double *bmod;
  // outputs of the energy pass
  double *forces;
  double4 *dEdd;
};

// ------------------------------------------------------------------ box and per-atom set-up
template <typename T>
__global__ void k_box(Dev<T> a, const double *boxes) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s == 0) { a.max_count[0] = 0; a.max_count[1] = 0; }  // the step's largest row counts start here
  if (s >= a.nsys) return;
  const double *H = boxes + 9 * s;
  BoxInfo &B = a.box[s];
  int changed = 0;
  for (int k = 0; k < 9; ++k) changed |= (B.H[k] != H[k]);
  double d = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) + H[2] * (H[3] * H[7] - H[4] * H[6]);
  double Hi[9];  // cofactor inverse (box.py:195-234)
  Hi[0] = (H[4] * H[8] - H[5] * H[7]) / d; Hi[1] = (H[2] * H[7] - H[1] * H[8]) / d; Hi[2] = (H[1] * H[5] - H[2] * H[4]) / d;
  Hi[3] = (H[5] * H[6] - H[3] * H[8]) / d; Hi[4] = (H[0] * H[8] - H[2] * H[6]) / d; Hi[5] = (H[2] * H[3] - H[0] * H[5]) / d;
  Hi[6] = (H[3] * H[7] - H[4] * H[6]) / d; Hi[7] = (H[1] * H[6] - H[0] * H[7]) / d; Hi[8] = (H[0] * H[4] - H[1] * H[3]) / d;
  for (int k = 0; k < 9; ++k) { B.H[k] = H[k]; B.Hinv[k] = Hi[k]; }
  B.vol = fabs(d);
  for (int c = 0; c < 3; ++c) B.idiag[c] = 1.0 / H[4 * c];
  const SysInfo &S = a.sys[s];
  for (int ax = 0; ax < 3; ++ax) {
    // plane height h_a = 1 / |column a of H^-1|
    double c0 = Hi[0 * 3 + ax], c1 = Hi[1 * 3 + ax], c2v = Hi[2 * 3 + ax];
    B.h[ax] = 1.0 / sqrt(c0 * c0 + c1 * c1 + c2v * c2v);
    int nc = S.nc[ax];
    int R = (int)ceil((a.cutoff + a.skin) * nc / B.h[ax] - 1e-12);
    B.R[ax] = (2 * R + 1 >= nc) ? -1 : R;
  }
  B.changed = changed;
  if (changed) atomicOr(a.nb_flag, 1);
  int bad = (fabs(H[1]) > 1e-12 * fabs(H[0])) || (fabs(H[2]) > 1e-12 * fabs(H[0])) || (fabs(H[5]) > 1e-12 * fabs(H[0])) ||
            !(H[0] > 0 && H[4] > 0 && H[8] > 0);
  double mc = 0.5 * fmin(H[0], fmin(H[4], H[8]));
  if (a.cutoff > mc) bad = 1;
  B.bad = bad;
  a.status[s] = bad ? 0x8u : 0u;  // the step's status word starts here
}

// Fractional coordinates, spline base and offset (pme.py:269-304), permanent dipoles
// (forcefield.py:1032-1042) and the cell of every atom.
template <typename T>
__global__ void k_prep(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  int s = a.sysid[i];
  const SysInfo &S = a.sys[s];
  const BoxInfo &B = a.box[s];
  double px = a.pos[3 * i], py = a.pos[3 * i + 1], pz = a.pos[3 * i + 2];
  double uc[3];
  int4 b;
  v4<T> f;
  int bb[3];
  T ff[3];
  bool finite = true;
  for (int ax = 0; ax < 3; ++ax) {
    double u = px * B.Hinv[0 * 3 + ax] + py * B.Hinv[1 * 3 + ax] + pz * B.Hinv[2 * 3 + ax];
    double fr = u - floor(u);
    if (!(fr >= 0.0 && fr < 1.0)) { fr = 0.0; finite = false; }  // non-finite position: keep indices in range
    uc[ax] = fr;
    double w = fr * S.K[ax];
    double fl = floor(w);
    int bv = (int)fl;
    if (bv >= S.K[ax]) bv -= S.K[ax];  // w rounded up to K: grid point K is point 0
    if (bv < 0) bv = 0;
    bb[ax] = bv;
    ff[ax] = T(w - fl);
  }
  if (!finite) atomicOr(&a.status[s], 0x4u);
  b.x = bb[0]; b.y = bb[1]; b.z = bb[2]; b.w = 0;
  f.x = ff[0]; f.y = ff[1]; f.z = ff[2]; f.w = T(0);
  a.base[i] = b;
  a.frac[i] = f;
  double4 p = make_double4(0, 0, 0, 0);
  if (a.perm) {
    for (int c = a.cov_start[i]; c < a.cov_start[i + 1]; ++c) {
      int j = a.cov_j[c];
      double vx = a.pos[3 * j] - px, vy = a.pos[3 * j + 1] - py, vz = a.pos[3 * j + 2] - pz;
      min_image(vx, vy, vz, B.H);
      double l = sqrt(vx * vx + vy * vy + vz * vz);
      double cc = a.cov_c[c] / l;
      p.x += cc * vx; p.y += cc * vy; p.z += cc * vz;
    }
  }
  a.pperm[i] = p;
  a.pos4[i] = make_double4(px, py, pz, (double)a.molid[i]);
  if (a.pos4f) {  // wrapped: |coordinates| below the box's, so FP32 keeps displacements to ~1e-6 nm
    double w[3];
    for (int c = 0; c < 3; ++c) w[c] = uc[0] * B.H[0 * 3 + c] + uc[1] * B.H[1 * 3 + c] + uc[2] * B.H[2 * 3 + c];
    a.pos4f[i] = make_float4(float(w[0]), float(w[1]), float(w[2]), float(a.molid[i]));
  }
  // Verlet list: rebuild when an atom moved more than skin / 2 since the last build
  double4 r0 = a.pos_ref[i];
  double dx = px - r0.x, dy = py - r0.y, dz = pz - r0.z;
  min_image(dx, dy, dz, B.H);
  double h2 = 0.25 * a.skin * a.skin;
  if (!(dx * dx + dy * dy + dz * dz <= h2)) atomicOr(a.nb_flag, 1);
  (void)uc;
}

// Cell of every atom (only when the candidate list is rebuilt).
template <typename T>
__global__ void k_cell_assign(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  if (!*a.nb_flag) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  int s = a.sysid[i];
  const SysInfo &S = a.sys[s];
  const BoxInfo &B = a.box[s];
  double4 p = a.pos4[i];
  double uc[3];
  for (int ax = 0; ax < 3; ++ax) {
    double u = p.x * B.Hinv[0 * 3 + ax] + p.y * B.Hinv[1 * 3 + ax] + p.z * B.Hinv[2 * 3 + ax];
    double fr = u - floor(u);
    if (!(fr >= 0.0 && fr < 1.0)) fr = 0.0;
    uc[ax] = fr;
  }
  int c0 = max(0, min((int)(uc[0] * S.nc[0]), S.nc[0] - 1));
  int c1 = max(0, min((int)(uc[1] * S.nc[1]), S.nc[1] - 1));
  int c2v = max(0, min((int)(uc[2] * S.nc[2]), S.nc[2] - 1));
  int cell = S.cell0 + (c0 * S.nc[1] + c1) * S.nc[2] + c2v;
  a.cell_of[i] = cell;
  a.slot_of[i] = atomicAdd(&a.cell_count[cell], 1);
}

// Offsets of every atom from its molecule's centre of mass (molecule made whole from its first
// atom), for the molecular virial.
template <typename T>
__global__ void k_mol(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmol) return;
  int i0 = a.mol_start[m], i1 = a.mol_start[m + 1];
  const BoxInfo &B = a.box[a.sysid[i0]];
  double cx = 0, cy = 0, cz = 0, mt = 0;
  for (int i = i0; i < i1; ++i) {
    double vx = a.pos[3 * i] - a.pos[3 * i0], vy = a.pos[3 * i + 1] - a.pos[3 * i0 + 1], vz = a.pos[3 * i + 2] - a.pos[3 * i0 + 2];
    min_image(vx, vy, vz, B.H);
    a.off[i] = make_double4(vx, vy, vz, 0);
    cx += a.mass[i] * vx; cy += a.mass[i] * vy; cz += a.mass[i] * vz; mt += a.mass[i];
  }
  cx /= mt; cy /= mt; cz /= mt;
  for (int i = i0; i < i1; ++i) {
    double4 o = a.off[i];
    a.off[i] = make_double4(o.x - cx, o.y - cy, o.z - cz, 0);
  }
}

// Exclusive scan of the cell counts of all systems (one block).
__global__ void k_scan_cells(const int *count, int *start, int n, const int *flag) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  if (!*flag) return;
  __shared__ int part[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    int i = base + threadIdx.x;
    int v = i < n ? count[i] : 0;
    part[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      int t = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
      __syncthreads();
      part[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n) start[i] = carry + part[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += part[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) start[n] = carry;
}

template <typename T>
__global__ void k_scatter(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  if (!*a.nb_flag) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  int t = a.cell_start[a.cell_of[i]] + a.slot_of[i];
  a.cell_atoms[t] = i;
  a.spos[t] = a.pos4[i];
}

// ------------------------------------------------------------------ Verlet candidate list
// One warp per atom when the list is rebuilt: every atom of another molecule within
// cutoff + skin, found through the cell list (cells within R along each axis), compacted by ballot;
// the positions of the build are kept for the displacement test (the reference's neighbour list,
// md/neighbors.py:169-304, rebuilt when an atom moved more than skin / 2).
template <typename T>
__global__ void __launch_bounds__(256) k_cand(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  if (!*a.nb_flag) return;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int s = a.wb_sys[blockIdx.x];
  int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  if (i >= S.atom0 + S.natom) return;
  const BoxInfo &B = a.box[s];
  double H[9], id[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) H[k] = B.H[k];
  id[0] = B.idiag[0]; id[1] = B.idiag[1]; id[2] = B.idiag[2];
  double4 pi = a.pos4[i];
  int mi = (int)pi.w;
  double rl = a.cutoff + a.skin, rl2 = rl * rl;
  int *out = a.cand + (size_t)i * a.cc;
  int count = 0;
  int cell = a.cell_of[i] - S.cell0;
  int n0 = S.nc[0], n1 = S.nc[1], n2 = S.nc[2];
  int ci2 = cell % n2, ci1 = (cell / n2) % n1, ci0 = cell / (n1 * n2);
  int R0 = B.R[0], R1 = B.R[1], R2 = B.R[2];
  int lo0 = R0 < 0 ? 0 : -R0, hi0 = R0 < 0 ? n0 - 1 : R0;
  int lo1 = R1 < 0 ? 0 : -R1, hi1 = R1 < 0 ? n1 - 1 : R1;
  for (int d0 = lo0; d0 <= hi0; ++d0) {
    int c0 = R0 < 0 ? d0 : ((ci0 + d0) % n0 + n0) % n0;
    for (int d1 = lo1; d1 <= hi1; ++d1) {
      int c1 = R1 < 0 ? d1 : ((ci1 + d1) % n1 + n1) % n1;
      int rowc = S.cell0 + (c0 * n1 + c1) * n2;
      int segs[2][2];
      int nseg = 0;
      if (R2 < 0) {
        segs[0][0] = 0; segs[0][1] = n2 - 1; nseg = 1;
      } else {
        int lo = ci2 - R2, hi = ci2 + R2;
        if (lo < 0) { segs[0][0] = lo + n2; segs[0][1] = n2 - 1; segs[1][0] = 0; segs[1][1] = hi; nseg = 2; }
        else if (hi >= n2) { segs[0][0] = lo; segs[0][1] = n2 - 1; segs[1][0] = 0; segs[1][1] = hi - n2; nseg = 2; }
        else { segs[0][0] = lo; segs[0][1] = hi; nseg = 1; }
      }
      for (int g = 0; g < nseg; ++g) {
        int a0 = a.cell_start[rowc + segs[g][0]], a1 = a.cell_start[rowc + segs[g][1] + 1];
        for (int t0 = a0; t0 < a1; t0 += 32) {
          int t = t0 + lane;
          bool keep = false;
          if (t < a1) {
            double4 pj = a.spos[t];
            if ((int)pj.w != mi) {
              double x = pi.x - pj.x, y = pi.y - pj.y, z = pi.z - pj.z;
              min_image_fast(x, y, z, H, id);
              keep = x * x + y * y + z * z < rl2;
            }
          }
          unsigned bal = __ballot_sync(0xffffffffu, keep);
          if (keep) {
            int slot = count + __popc(bal & ((1u << lane) - 1u));
            if (slot < a.cc) out[slot] = a.cell_atoms[t];
          }
          count += __popc(bal);
        }
      }
    }
  }
  if (lane == 0) {
    a.ncand[i] = count;
    a.pos_ref[i] = pi;
    if (count > a.cc) atomicOr(&a.status[s], 0x10u);
  }
}

// End of a rebuild: clear the cell counts for the next one, count it, lower the flag.
__global__ void k_nb_finish(int *cell_count, int ncell, int *flag, long long *builds) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  if (!*flag) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += gridDim.x * blockDim.x) cell_count[c] = 0;
}
__global__ void k_nb_lower(int *flag, long long *builds) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  if (*flag) { *flag = 0; *builds += 1; }
}

// ------------------------------------------------------------------ pair rows
// k_rows: one warp per atom finds the row -- the molecule partners (always kept inside the cutoff;
// the rigid special table of md/topology.py:161-178), then the candidates of the Verlet list (or
// the caller's rows), masked to r < rc (forcefield.py:1140-1195) -- and writes k, x, y, z compacted
// by ballot; then the same warp evaluates the radial kernels G_n = B_n[erf(a r)/r] -
// B_n[erf(beta r)/r] (forcefield.py:1314-1338, kernels.py:76-118) of its row's entries from the
// rounded displacements it stored, every lane busy, and writes with them the local
// preconditioner's short entries and the learned guess's graph edges.

// An atom's group of LPA lanes (32: the warp; 16, 8: a half, a quarter warp): its shuffle mask, and the sum over
// it (the warp's own reduction for a whole warp).
template <int LPA>
__device__ __forceinline__ unsigned group_mask() {
  if constexpr (LPA == 32) return 0xffffffffu;
  else return ((1u << LPA) - 1u) << ((threadIdx.x & 31) & ~(LPA - 1));
}
template <typename T, int LPA>
__device__ __forceinline__ T group_sum(T v, unsigned m) {
  if constexpr (LPA == 32) {
    return warp_sum<T>(v);
  } else {
#pragma unroll
    for (int o = LPA / 2; o > 0; o >>= 1) v += __shfl_xor_sync(m, v, o);
    return v;
  }
}

// FP32 sequential minimum image (the mixed-precision row build's candidate loop).
__device__ __forceinline__ void min_image_fast_f(float &x, float &y, float &z, const float *H, const float *id) {
  float n = rintf(z * id[2]);
  x -= n * H[6]; y -= n * H[7]; z -= n * H[8];
  n = rintf(y * id[1]);
  x -= n * H[3]; y -= n * H[4];
  n = rintf(x * id[0]);
  x -= n * H[0];
}

// The row scan of atom i by its group of LPA lanes: the molecule partners (special = true), then the
// candidates, one entry per lane and round, the next round's candidate loaded before the current one
// is tested.  visit(keep, j, x, y, z, special) runs on all LPA lanes every round (it may use the
// group's collectives);
// keep is r < rc for an entry of another atom, false on lanes without one; the displacement comes
// as T, as the rows store it.  Mixed precision: the candidates' FP32 displacements from the wrapped
// FP32 positions (16-byte gathers), the molecule partners' rounded from FP64.
template <typename T, int LPA, typename Visit>
__device__ __forceinline__ void row_scan(const Dev<T> &a, const SysInfo &S, const BoxInfo &B, int i, int lane, Visit &&visit) {
  double H[9], id[3];
#pragma unroll
  for (int k = 0; k < 9; ++k) H[k] = B.H[k];
  id[0] = B.idiag[0]; id[1] = B.idiag[1]; id[2] = B.idiag[2];
  const double4 pi = a.pos4[i];
  const double rc2 = a.cutoff * a.cutoff;
  const int mf = a.molfirst[i], me = a.molend[i];
  for (int j0 = mf; j0 < me; j0 += LPA) {
    int j = j0 + lane;
    bool keep = false;
    double x = 0, y = 0, z = 0;
    if (j < me && j != i) {
      double4 pj = a.pos4[j];
      x = pi.x - pj.x; y = pi.y - pj.y; z = pi.z - pj.z;
      min_image_fast(x, y, z, H, id);
      keep = x * x + y * y + z * z < rc2;
    }
    visit(keep, j, T(x), T(y), T(z), true);
  }
  const int mi = (int)pi.w;
  const int *row;
  int nc;
  if (a.idx) {  // the caller's candidate rows (local indices, padding natom)
    row = a.idx + (size_t)i * a.idx_width;
    nc = a.idx_width;
  } else {      // the engine's Verlet candidates (within cutoff + skin at the last rebuild)
    row = a.cand + (size_t)i * a.cc;
    nc = min(a.ncand[i], a.cc);
  }
  auto partner = [&](int c) {
    int j = -1;
    if (c < nc) {
      int jl = row[c];
      if (a.idx) j = (jl >= 0 && jl < S.natom) ? S.atom0 + jl : -1;
      else j = jl;
    }
    return j;
  };
  if (sizeof(T) == 4 && a.pos4f) {
    float Hf[9], idf[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) Hf[k] = float(H[k]);
    idf[0] = float(id[0]); idf[1] = float(id[1]); idf[2] = float(id[2]);
    const float4 pf = a.pos4f[i];
    const float rc2f = float(rc2);
    int jn = partner(lane);
    float4 pn = jn >= 0 ? a.pos4f[jn] : make_float4(0.f, 0.f, 0.f, -1.f);
    for (int c0 = 0; c0 < nc; c0 += LPA) {
      const int j = jn;
      const float4 pj = pn;
      jn = partner(c0 + LPA + lane);  // prefetch the next round
      if (jn >= 0) pn = a.pos4f[jn];
      bool keep = false;
      float x = 0.f, y = 0.f, z = 0.f;
      if (j >= 0 && (int)pj.w != mi) {
        x = pf.x - pj.x; y = pf.y - pj.y; z = pf.z - pj.z;
        min_image_fast_f(x, y, z, Hf, idf);
        keep = x * x + y * y + z * z < rc2f;
      }
      visit(keep, j, x, y, z, false);
    }
  } else {
    int jn = partner(lane);
    double4 pn = jn >= 0 ? a.pos4[jn] : make_double4(0, 0, 0, -1);
    for (int c0 = 0; c0 < nc; c0 += LPA) {
      const int j = jn;
      const double4 pj = pn;
      jn = partner(c0 + LPA + lane);  // prefetch the next round
      if (jn >= 0) pn = a.pos4[jn];
      bool keep = false;
      double x = 0, y = 0, z = 0;
      if (j >= 0 && (int)pj.w != mi) {
        x = pi.x - pj.x; y = pi.y - pj.y; z = pi.z - pj.z;
        min_image_fast(x, y, z, H, id);
        keep = x * x + y * y + z * z < rc2;
      }
      visit(keep, j, T(x), T(y), T(z), false);
    }
  }
}

template <typename T, bool EVAL>
__device__ __forceinline__ void row_keep(const Dev<T> &a, bool keep, int j, T x, T y, T z, size_t base, int &count, unsigned gm,
                                         int i, T Ri, int &ecount, int &vcount, int &scount, bool special) {
  const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;  // the lanes below this one (the group's bits only
                                                          // are set in its ballots)
  const T r2 = x * x + y * y + z * z;  // the tests below in the rows' precision
  bool kv = false;
  if (a.rnv && keep && !(r2 < T(a.rce2))) {  // split rows: beyond elec_cutoff only pairs with an LJ term stay
    kv = !special && j >= 0 && a.seps[i] * a.seps[j] != T(0);  // molecule partners have LJ weight 0
    keep = false;
  }
  // the slots first (all lanes take part in the ballots), then one branch for an entry's stores
  const unsigned bal = __ballot_sync(gm, keep);
  const int slot = count + __popc(bal & lt);
  count += __popc(bal);
  const bool kept = keep && slot < a.mce;
  if constexpr (!EVAL) {  // the entry alone; its kernels, short entry and edge follow the scan
    if (kept) {
      const size_t o = base + slot;
      a.rk[o] = j;
      a.rx[o] = x; a.ry[o] = y; a.rz[o] = z;
    }
  } else {
  bool sh = false, ed = false;
  int at_s = 0, at_e = 0;
  if (a.sh_n) {  // the local preconditioner's entries: partner, displacement, G1, G2, entry-major
    sh = kept && r2 < T(a.lc2);
    const unsigned sb = __ballot_sync(gm, sh);
    at_s = scount + __popc(sb & lt);
    scount += __popc(sb);
    sh = sh && at_s < a.sh_max;
  }
  if (a.nn_e4) {  // the learned guess's graph edges: the entries closer than rg, with G1, G2
    ed = kept && float(r2) < a.nn_rg2;
    const unsigned eb = __ballot_sync(gm, ed);
    at_e = ecount + __popc(eb & lt);
    ecount += __popc(eb);
    ed = ed && at_e < a.nn_emax;
  }
  if (kept) {
    const size_t o = base + slot;
    a.rk[o] = j;
    a.rx[o] = x; a.ry[o] = y; a.rz[o] = z;
    const T r = t_sqrt(r2), Rk = a.radius[j];
    const T aik = t_rsqrt(T(2) * (Ri * Ri + Rk * Rk));
    T A[4], Bb[4];
    erf_kernels<T>(aik, r, A);
    erf_kernels<T>(T(a.beta), r, Bb);
    const T g1 = A[1] - Bb[1], g2 = A[2] - Bb[2];
    a.rg0[o] = A[0] - Bb[0]; a.rg1[o] = g1; a.rg2[o] = g2; a.rg3[o] = A[3] - Bb[3];
    if (sh) {
      const size_t c = (size_t)at_s * a.nt + i;
      a.c_k[c] = j;
      a.c_x[c] = x; a.c_y[c] = y; a.c_z[c] = z;
      a.c_g1[c] = g1; a.c_g2[c] = g2;
    }
    if (ed) {
      const size_t e = (size_t)i * a.nn_emax + at_e;
      a.nn_e4[e] = make_float4(float(x), float(y), float(z), __int_as_float(j));
      a.nn_g[e] = make_float2(float(g1), float(g2));
    }
  }
  }
  if (a.rnv) {
    const unsigned bv = __ballot_sync(gm, kv);
    const int sv = vcount + __popc(bv & lt);
    if (kv && sv < a.mc - a.mce) {
      const size_t o = base + a.mce + sv;
      a.rk[o] = j;
      a.rx[o] = x; a.ry[o] = y; a.rz[o] = z;
    }
    vcount += __popc(bv);
  }
}

// TWO_PHASE: the scan stores the entries only; then the group evaluates the kernels of its row
// (read back from L2) with every lane busy, and assigns the short entries and graph edges in row order.
template <typename T, int LPA = 32, bool TWO_PHASE = false>
__global__ void __launch_bounds__(8 * LPA, 6 * 32 / LPA) k_rows(Dev<T> a) {
  static_assert(LPA == 32 || LPA == 16 || LPA == 8, "lanes per atom");
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  const int warp = threadIdx.x / LPA, lane = threadIdx.x % LPA;  // the atom's group of LPA lanes
  const unsigned gm = group_mask<LPA>();
  const int s = a.wb_sys[blockIdx.x];
  const int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  if (i >= S.atom0 + S.natom) return;
  const T Ri = a.radius[i];
  const size_t base = (size_t)i * a.mc;
  int count = 0, ecount = 0, vcount = 0, scount = 0, nsp = 0;
  row_scan<T, LPA>(a, S, a.box[s], i, lane, [&](bool keep, int j, T x, T y, T z, bool special) {
    row_keep<T, !TWO_PHASE>(a, keep, j, x, y, z, base, count, gm, i, Ri, ecount, vcount, scount, special);
    if (special) nsp = count;
  });
  if constexpr (TWO_PHASE) {
    __syncwarp(gm);  // the row, stored by the group's lanes, visible to all of them
    const unsigned lt = (1u << (threadIdx.x & 31)) - 1u;
    const int n = min(count, a.mce);
    const T beta = T(a.beta), lc2 = T(a.lc2);
    // the next round's entry is loaded before the current one is evaluated
    auto load = [&](int t, int &j, T &x, T &y, T &z) {
      const bool in = t < n;
      const size_t o = base + (in ? t : 0);
      j = in ? a.rk[o] : 0;
      x = in ? a.rx[o] : T(0); y = in ? a.ry[o] : T(0); z = in ? a.rz[o] : T(0);
    };
    int jn;
    T xn, yn, zn;
    load(lane, jn, xn, yn, zn);
    for (int t0 = 0; t0 < n; t0 += LPA) {
      const int t = t0 + lane;
      const bool in = t < n;
      const size_t o = base + (in ? t : 0);
      const int j = jn;
      const T x = xn, y = yn, z = zn;
      load(t + LPA, jn, xn, yn, zn);
      const T r2 = x * x + y * y + z * z;
      bool sh = false, ed = false;
      int at_s = 0, at_e = 0;
      if (a.sh_n) {  // the local preconditioner's entries: partner, displacement, G1, G2, entry-major
        sh = in && r2 < lc2;
        const unsigned sb = __ballot_sync(gm, sh);
        at_s = scount + __popc(sb & lt);
        scount += __popc(sb);
        sh = sh && at_s < a.sh_max;
      }
      if (a.nn_e4) {  // the learned guess's graph edges: the entries closer than rg, with G1, G2
        ed = in && float(r2) < a.nn_rg2;
        const unsigned eb = __ballot_sync(gm, ed);
        at_e = ecount + __popc(eb & lt);
        ecount += __popc(eb);
        ed = ed && at_e < a.nn_emax;
      }
      if (in) {
        const T r = t_sqrt(r2), Rk = a.radius[j];
        const T aik = t_rsqrt(T(2) * (Ri * Ri + Rk * Rk));
        T A[4], Bb[4];
        erf_kernels<T>(aik, r, A);
        erf_kernels<T>(beta, r, Bb);
        const T g1 = A[1] - Bb[1], g2 = A[2] - Bb[2];
        a.rg0[o] = A[0] - Bb[0]; a.rg1[o] = g1; a.rg2[o] = g2; a.rg3[o] = A[3] - Bb[3];
        if (sh) {
          const size_t c = (size_t)at_s * a.nt + i;
          a.c_k[c] = j;
          a.c_x[c] = x; a.c_y[c] = y; a.c_z[c] = z;
          a.c_g1[c] = g1; a.c_g2[c] = g2;
        }
        if (ed) {
          const size_t e = (size_t)i * a.nn_emax + at_e;
          a.nn_e4[e] = make_float4(float(x), float(y), float(z), __int_as_float(j));
          a.nn_g[e] = make_float2(float(g1), float(g2));
        }
      }
    }
  }
  if (lane == 0) {
    a.rn[i] = count;
    a.rnsp[i] = nsp;
    if (a.nn_e4) a.nn_ne[i] = ecount;
    if (a.sh_n) {
      a.sh_n[i] = min(scount, a.sh_max);
      if (scount > a.sh_max) atomicOr(&a.status[s], 0x20u);  // the preconditioner kept the first sh_max
    }
    if (count > a.mce) atomicOr(&a.status[s], 0x1u);
    atomicMax(a.max_count, count);
    if (a.rnv) {
      a.rnv[i] = vcount;
      if (vcount > a.mc - a.mce) atomicOr(&a.status[s], 0x1u);
      atomicMax(a.max_count + 1, vcount);
    }
  }
}

// ------------------------------------------------------------------ PME influence function
// G(m) = exp(-pi^2 |m*|^2 / beta^2) / (2 pi V |m*|^2) / (b1 b2 b3), 0 at m = 0 (pme.py:243-267),
// on the half spectrum, computed in FP64, stored in T; recomputed only when the box changed.
template <typename T>
__global__ void k_influence(Dev<T> a, long long total) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
    int s = 0;
    while (s + 1 < a.nsys && a.sys[s + 1].cgrid0 <= g) ++s;
    const SysInfo &S = a.sys[s];
    const BoxInfo &B = a.box[s];
    if (!B.changed) continue;
    long long l = g - S.cgrid0;
    if (l >= (long long)S.K[0] * S.K[1] * S.K3h) continue;  // alignment gap between systems
    int m3 = (int)(l % S.K3h);
    long long t = l / S.K3h;
    int k2 = (int)(t % S.K[1]), k1 = (int)(t / S.K[1]);
    int m1 = k1 <= (S.K[0] - 1) / 2 ? k1 : k1 - S.K[0];
    int m2 = k2 <= (S.K[1] - 1) / 2 ? k2 : k2 - S.K[1];
    if (S.K[0] % 2 == 0 && k1 == S.K[0] / 2) m1 = -S.K[0] / 2;
    if (S.K[1] % 2 == 0 && k2 == S.K[1] / 2) m2 = -S.K[1] / 2;
    double mv[3];
    for (int c = 0; c < 3; ++c) mv[c] = m1 * B.Hinv[c * 3 + 0] + m2 * B.Hinv[c * 3 + 1] + m3 * B.Hinv[c * 3 + 2];
    double msq = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
    double G = 0.0;
    if (msq > 0) {
      G = exp(-PI * PI * msq / (a.beta * a.beta)) / (2.0 * PI * B.vol * msq);
      G /= a.bmod[S.mod0[0] + k1] * a.bmod[S.mod0[1] + k2] * a.bmod[S.mod0[2] + m3];
    }
    a.Ginf[g] = T(G);
  }
}

// ------------------------------------------------------------------ spread (pme.py:306-337)
// A group of LPA lanes per atom (a warp, or 16 / 8 lanes: two or four atoms per warp, whose B-spline
// weights, stencil rounds and tails proceed together), the P^3 stencil over the group's lanes, atomic
// adds into the system's grid.  With UPDATE_P the CG direction is first advanced, p = z + beta p
// (forcefield.py:1812), and spread.
template <typename T, int P, bool WITH_Q, bool UPDATE_P, int ACT, int LPA = 32>
__global__ void __launch_bounds__(8 * LPA) k_spread(Dev<T> a, const v4<T> *__restrict__ vin) {
  static_assert(LPA == 32 || LPA == 16 || LPA == 8 || LPA == 4, "lanes per atom");
  pdl_enter();
  __shared__ T sh[WARPS_PER_BLOCK][2][3][P];  // per atom of the block
  const int warp = threadIdx.x / LPA, lane = threadIdx.x % LPA;  // the atom's group of LPA lanes
  const unsigned gm = group_mask<LPA>();
  int s = a.wb_sys[blockIdx.x];
  int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  if (i >= S.atom0 + S.natom) return;
  if (ACT == 1 && !a.cg[s].active) return;
  if (ACT == 2 && !a.cg[s].sweep2) return;
  if (ACT == 3 && !a.cg[s].fallback) return;
  v4<T> d;
  if (UPDATE_P) {
    v4<T> z = a.Z[i], p = a.P[i];
    T bt = T(a.cg[s].beta);
    d.x = z.x + bt * p.x; d.y = z.y + bt * p.y; d.z = z.z + bt * p.z; d.w = T(0);
    __syncwarp(gm);
    if (lane == 0) a.P[i] = d;
  } else {
    d = vin[i];
  }
  const BoxInfo &B = a.box[s];
  int4 b = a.base[i];
  v4<T> f = a.frac[i];
  if (lane < 3) {
    T th[P], dth[P];
    bspline<T, P, false>(lane == 0 ? f.x : (lane == 1 ? f.y : f.z), th, dth, nullptr);
#pragma unroll
    for (int k = 0; k < P; ++k) { sh[warp][0][lane][k] = th[k]; sh[warp][1][lane][k] = dth[k]; }
  }
  __syncwarp(gm);
  T e[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax)
    e[ax] = T((double(d.x) * B.Hinv[0 * 3 + ax] + double(d.y) * B.Hinv[1 * 3 + ax] + double(d.z) * B.Hinv[2 * 3 + ax]) * S.K[ax]);
  T qi = WITH_Q ? a.q[i] : T(0);
  T *grid = a.Q + S.rgrid0;
  const int K1 = S.K[0], K2 = S.K[1], K3 = S.K[2];
  if constexpr (sizeof(T) == 4) {
    if ((K3 & 3) == 0 && (S.rgrid0 & 3) == 0) {
      // 16-byte vector reductions: along k3 the P points of a stencil row fall into ng aligned
      // groups of 4 (2.4x fewer L2 atomic operations than one per point); the weight of a point is
      // A(j1, j2) t3 + B(j1, j2) u3 with A = (q t1 + e1 u1) t2 + e2 t1 u2, B = e3 t1 t2.
      const int g0 = b.z >> 2, ng = ((b.z + P - 1) >> 2) - g0 + 1, K34 = K3 >> 2;
      for (int sl = lane; sl < P * P * ng; sl += LPA) {
        int r = ng == 2 ? (sl >> 1) : (ng == 3 ? sl / 3 : sl / ng), gi = sl - r * ng;  // no runtime division for 2, 3
        int j1 = r / P, j2 = r - j1 * P;
        T t1 = sh[warp][0][0][j1], t2 = sh[warp][0][1][j2];
        T u1 = sh[warp][1][0][j1], u2 = sh[warp][1][1][j2];
        T A = (qi * t1 + e[0] * u1) * t2 + e[1] * t1 * u2, Bw = e[2] * t1 * t2;
        int g = g0 + gi;
        float vv[4];
#pragma unroll
        for (int el = 0; el < 4; ++el) {
          int j3 = 4 * g + el - b.z;
          vv[el] = (j3 >= 0 && j3 < P) ? A * sh[warp][0][2][j3] + Bw * sh[warp][1][2][j3] : 0.0f;
        }
        int i1 = b.x + j1; if (i1 >= K1) i1 -= K1;
        int i2 = b.y + j2; if (i2 >= K2) i2 -= K2;
        int gp = g >= K34 ? g - K34 : g;
        atomicAdd(reinterpret_cast<float4 *>(grid + ((size_t)i1 * K2 + i2) * K3) + gp, make_float4(vv[0], vv[1], vv[2], vv[3]));
      }
      return;
    }
  }
  for (int p = lane; p < P * P * P; p += LPA) {
    int j1 = p / (P * P), j2 = (p / P) % P, j3 = p % P;
    T t1 = sh[warp][0][0][j1], t2 = sh[warp][0][1][j2], t3 = sh[warp][0][2][j3];
    T u1 = sh[warp][1][0][j1], u2 = sh[warp][1][1][j2], u3 = sh[warp][1][2][j3];
    T v = (qi * t1 + e[0] * u1) * t2 * t3 + e[1] * t1 * u2 * t3 + e[2] * t1 * t2 * u3;
    int i1 = b.x + j1; if (i1 >= K1) i1 -= K1;
    int i2 = b.y + j2; if (i2 >= K2) i2 -= K2;
    int i3 = b.z + j3; if (i3 >= K3) i3 -= K3;
    atomicAdd(grid + ((size_t)i1 * K2 + i2) * K3 + i3, v);
  }
}

// ------------------------------------------------------------------ FFT (shared memory, Stockham)
template <typename T>
__device__ __forceinline__ c2<T> cmul(c2<T> a, c2<T> b) {
  c2<T> r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// Compile-time radix plan of a length-L transform: radix 8 first, then 4, 2, 3, 5 (the runtime
// plans of the host use 4, 2, 3, 5).
__host__ __device__ constexpr int fft_nst(int L) {
  int n = 0;
  while (L % 8 == 0) { L /= 8; ++n; }
  while (L % 4 == 0) { L /= 4; ++n; }
  while (L % 2 == 0) { L /= 2; ++n; }
  while (L % 3 == 0) { L /= 3; ++n; }
  while (L % 5 == 0) { L /= 5; ++n; }
  return n;
}
__host__ __device__ constexpr int fft_radix(int L, int st) {
  int n = 0;
  while (L % 8 == 0) { if (n == st) return 8; L /= 8; ++n; }
  while (L % 4 == 0) { if (n == st) return 4; L /= 4; ++n; }
  while (L % 2 == 0) { if (n == st) return 2; L /= 2; ++n; }
  while (L % 3 == 0) { if (n == st) return 3; L /= 3; ++n; }
  while (L % 5 == 0) { if (n == st) return 5; L /= 5; ++n; }
  return 1;
}

// R-point DFT in registers, sign -1 forward / +1 inverse: X_k = sum_n v_n w^(n k), w = exp(sign 2 pi i / R).
template <typename T, int R>
__device__ __forceinline__ void butterfly(c2<T> *v, T sg) {
  c2<T> o[R];
  if constexpr (R == 8) {
    // two 4-point DFTs of the even and odd points, X_k = E_k + w^k O_k, X_(k+4) = E_k - w^k O_k
    c2<T> e[4] = {v[0], v[2], v[4], v[6]}, d[4] = {v[1], v[3], v[5], v[7]};
    butterfly<T, 4>(e, sg);
    butterfly<T, 4>(d, sg);
    const T h = T(0.70710678118654752440);
    c2<T> t[4];
    t[0] = d[0];
    t[1].x = h * (d[1].x - sg * d[1].y); t[1].y = h * (d[1].y + sg * d[1].x);
    t[2].x = -sg * d[2].y; t[2].y = sg * d[2].x;
    t[3].x = -h * (d[3].x + sg * d[3].y); t[3].y = h * (sg * d[3].x - d[3].y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      o[k].x = e[k].x + t[k].x; o[k].y = e[k].y + t[k].y;
      o[k + 4].x = e[k].x - t[k].x; o[k + 4].y = e[k].y - t[k].y;
    }
  } else if constexpr (R == 2) {
    o[0].x = v[0].x + v[1].x; o[0].y = v[0].y + v[1].y;
    o[1].x = v[0].x - v[1].x; o[1].y = v[0].y - v[1].y;
  } else if constexpr (R == 4) {
    c2<T> a0, a1, b0, b1, ib1;
    a0.x = v[0].x + v[2].x; a0.y = v[0].y + v[2].y;
    a1.x = v[0].x - v[2].x; a1.y = v[0].y - v[2].y;
    b0.x = v[1].x + v[3].x; b0.y = v[1].y + v[3].y;
    b1.x = v[1].x - v[3].x; b1.y = v[1].y - v[3].y;
    ib1.x = -sg * b1.y; ib1.y = sg * b1.x;  // sign * i * b1
    o[0].x = a0.x + b0.x; o[0].y = a0.y + b0.y;
    o[2].x = a0.x - b0.x; o[2].y = a0.y - b0.y;
    o[1].x = a1.x + ib1.x; o[1].y = a1.y + ib1.y;
    o[3].x = a1.x - ib1.x; o[3].y = a1.y - ib1.y;
  } else if constexpr (R == 3) {
    const T c = T(-0.5), sn = sg * T(0.86602540378443864676);
    c2<T> t1, t2, m;
    t1.x = v[1].x + v[2].x; t1.y = v[1].y + v[2].y;
    t2.x = v[1].x - v[2].x; t2.y = v[1].y - v[2].y;
    o[0].x = v[0].x + t1.x; o[0].y = v[0].y + t1.y;
    m.x = v[0].x + c * t1.x; m.y = v[0].y + c * t1.y;
    o[1].x = m.x - sn * t2.y; o[1].y = m.y + sn * t2.x;
    o[2].x = m.x + sn * t2.y; o[2].y = m.y - sn * t2.x;
  } else {
    static_assert(R == 5, "radix");
    const T c1 = T(0.30901699437494742410), c2v = T(-0.80901699437494742410);
    const T s1 = sg * T(0.95105651629515357212), s2 = sg * T(0.58778525229247312917);
    c2<T> a1, a2, b1, b2, m1, m2, n1, n2;
    a1.x = v[1].x + v[4].x; a1.y = v[1].y + v[4].y;
    b1.x = v[1].x - v[4].x; b1.y = v[1].y - v[4].y;
    a2.x = v[2].x + v[3].x; a2.y = v[2].y + v[3].y;
    b2.x = v[2].x - v[3].x; b2.y = v[2].y - v[3].y;
    o[0].x = v[0].x + a1.x + a2.x; o[0].y = v[0].y + a1.y + a2.y;
    m1.x = v[0].x + c1 * a1.x + c2v * a2.x; m1.y = v[0].y + c1 * a1.y + c2v * a2.y;
    m2.x = v[0].x + c2v * a1.x + c1 * a2.x; m2.y = v[0].y + c2v * a1.y + c1 * a2.y;
    n1.x = s1 * b1.x + s2 * b2.x; n1.y = s1 * b1.y + s2 * b2.y;
    n2.x = s2 * b1.x - s1 * b2.x; n2.y = s2 * b1.y - s1 * b2.y;
    o[1].x = m1.x - n1.y; o[1].y = m1.y + n1.x;
    o[4].x = m1.x + n1.y; o[4].y = m1.y - n1.x;
    o[2].x = m2.x - n2.y; o[2].y = m2.y + n2.x;
    o[3].x = m2.x + n2.y; o[3].y = m2.y - n2.x;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = o[r];
}

// One Stockham stage (radix R, NS points already combined) of nl lines of length L in shared
// memory: v_r = x[j + r L/R] w^(r k), k = j mod NS, DFT_R, y[(j / NS) NS R + k + r NS].  LF (lines
// fastest): consecutive threads take the same j of consecutive lines, for line strides ld that are
// odd in 8-byte words, where the stride-R writes of the first stage would otherwise hit the same
// shared-memory banks; otherwise consecutive threads take consecutive j of one line.
template <typename T, int R, bool LF = false>
__device__ __forceinline__ void fft_stage(const c2<T> *x, c2<T> *y, int L, int NS, int nl, int ld, const c2<T> *tw, int sign) {
  const int LR = L / R, stride = L / (NS * R);
  const T sg = T(sign);
  for (int w = threadIdx.x; w < LR * nl; w += blockDim.x) {
    int line, j;
    if (LF) { j = w / nl; line = w - j * nl; }
    else { line = w / LR; j = w - line * LR; }
    int k = j % NS;
    const c2<T> *in = x + line * ld;
    c2<T> *out = y + line * ld;
    c2<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      c2<T> u = in[j + r * LR];
      if (r > 0) {
        c2<T> t = tw[r * k * stride];
        if (sign > 0) t.y = -t.y;
        u = cmul<T>(u, t);
      }
      v[r] = u;
    }
    butterfly<T, R>(v, sg);
    int dst = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[dst + r * NS] = v[r];
  }
  __syncthreads();
}

// Compile-time length: every index constant folds (L, R, NS template-known).
template <typename T, int L, int ST, int NS, bool LF = false>
__device__ __forceinline__ c2<T> *fft_run_ct(c2<T> *x, c2<T> *y, int nl, int ld, const c2<T> *tw, int sign) {
  if constexpr (ST == fft_nst(L)) {
    return x;
  } else {
    constexpr int R = fft_radix(L, ST);
    fft_stage<T, R, LF>(x, y, L, NS, nl, ld, tw, sign);
    return fft_run_ct<T, L, ST + 1, NS * R, LF>(y, x, nl, ld, tw, sign);
  }
}

// Runtime length (fallback for meshes without a compiled plan).
template <typename T>
__device__ c2<T> *fft_run_rt(c2<T> *x, c2<T> *y, int L, int nl, int ld, const int *rad, int nst, const c2<T> *tw, int sign) {
  int NS = 1;
  for (int st = 0; st < nst; ++st) {
    const int R = rad[st];
    if (R == 4) fft_stage<T, 4>(x, y, L, NS, nl, ld, tw, sign);
    else if (R == 2) fft_stage<T, 2>(x, y, L, NS, nl, ld, tw, sign);
    else if (R == 3) fft_stage<T, 3>(x, y, L, NS, nl, ld, tw, sign);
    else fft_stage<T, 5>(x, y, L, NS, nl, ld, tw, sign);
    c2<T> *t = x; x = y; y = t;
    NS *= R;
  }
  return x;
}

template <typename T, int L, bool LF = false>
__device__ __forceinline__ c2<T> *fft_lines(c2<T> *x, c2<T> *y, int Lrt, int nl, int ld, const int *rad, int nst, const c2<T> *tw,
                                            int sign) {
  if constexpr (L == 0) return fft_run_rt<T>(x, y, Lrt, nl, ld, rad, nst, tw, sign);
  else return fft_run_ct<T, L, 0, 1, LF>(x, y, nl, ld, tw, sign);
}

// Global -> shared staging of `total` elements by the FFT_THREADS threads of a pass: with a
// compile-time bound N every load of a thread is issued before its first store (the passes are
// latency-bound; one L2 round trip instead of one per element); N = 0: a plain loop.
template <int N, typename Get, typename Put>
__device__ __forceinline__ void staged_copy(int total, Get &&get, Put &&put) {
  if constexpr (N > 0) {
    constexpr int PER = (N + FFT_THREADS - 1) / FFT_THREADS;
    using V = decltype(get(0));
    V v[PER];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int t = threadIdx.x + j * FFT_THREADS;
      if (t < total) v[j] = get(t);
    }
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int t = threadIdx.x + j * FFT_THREADS;
      if (t < total) put(t, v[j]);
    }
  } else {
    for (int t = threadIdx.x; t < total; t += blockDim.x) put(t, get(t));
  }
}

template <typename T>
struct c2pair {
  c2<T> a, b;
};

static_assert(FFT_THREADS <= 256, "the FFT passes are compiled for at most 256 threads per CTA");

// A launch of an FFT pass covers a group of systems with the same mesh length along the pass's
// axis: block -> (group member g, tile) by the tile prefix gtile0 (ng + 1 entries).
__device__ __forceinline__ int group_member(const int *gtile0, int ng, int b) {
  int g = 0;
  while (g + 1 < ng && gtile0[g + 1] <= b) ++g;
  return g;
}

template <typename T>
__device__ __forceinline__ bool pass_active(const Dev<T> &a, int s, int act) {
  return act == 0 || (act == 1 && a.cg[s].active) || (act == 2 && a.cg[s].sweep2) || (act == 3 && a.cg[s].fallback);
}

// k3 pass, real -> half complex: two real lines packed as one complex line (z = a + i b), one
// length-K3 FFT, untangled.
template <typename T, int L>
__global__ void __launch_bounds__(256) k_fft_x_fwd(Dev<T> a, const int *gsys, const int *gtile0, int ng, int act) {
  pdl_enter();
  extern __shared__ unsigned char smem_raw[];
  int g = group_member(gtile0, ng, blockIdx.x);
  int s = gsys[g];
  if (!pass_active(a, s, act)) return;
  const SysInfo &S = a.sys[s];
  const int K3 = L ? L : S.K[2], K3h = K3 / 2 + 1, nlines = S.K[0] * S.K[1];
  int tile = blockIdx.x - gtile0[g];
  int l0 = tile * 2 * FFT_PAIRS;  // first real line
  int np = min(FFT_PAIRS, (nlines - l0) / 2);
  c2<T> *x = reinterpret_cast<c2<T> *>(smem_raw), *y = x + FFT_PAIRS * K3, *tws = y + FFT_PAIRS * K3;
  T *Q = a.Q + S.rgrid0 + (size_t)l0 * K3;
  for (int t = threadIdx.x; t < K3; t += blockDim.x) tws[t] = a.tw[S.tw[2] + t];  // twiddles in shared memory
  staged_copy<2 * FFT_PAIRS * L>(
      2 * np * K3, [&](int t) { return Q[t]; },
      [&](int t, T v) {
        int rl = t / K3, k = t - rl * K3;
        reinterpret_cast<T *>(&x[(rl >> 1) * K3 + k])[rl & 1] = v;
      });
  __syncthreads();
  c2<T> *res = fft_lines<T, L>(x, y, K3, np, K3, S.rad[2], S.nst[2], tws, -1);
  c2<T> *C = a.C + S.cgrid0 + (size_t)l0 * K3h;
  for (int t = threadIdx.x; t < np * K3h; t += blockDim.x) {
    int cl = t / K3h, m = t - cl * K3h;
    c2<T> Z = res[cl * K3 + m], W = res[cl * K3 + (m == 0 ? 0 : K3 - m)];
    c2<T> A, Bv;
    A.x = T(0.5) * (Z.x + W.x); A.y = T(0.5) * (Z.y - W.y);
    T dx = Z.x - W.x, dy = Z.y + W.y;  // (Z - conj W) / (2 i)
    Bv.x = T(0.5) * dy; Bv.y = -T(0.5) * dx;
    C[(size_t)(2 * cl) * K3h + m] = A;
    C[(size_t)(2 * cl + 1) * K3h + m] = Bv;
  }
}

// k3 pass, half complex -> real (the inverse of k_fft_x_fwd, unnormalised): writes phi.
template <typename T, int L>
__global__ void __launch_bounds__(256) k_fft_x_inv(Dev<T> a, const int *gsys, const int *gtile0, int ng, int act) {
  pdl_enter();
  extern __shared__ unsigned char smem_raw[];
  int g = group_member(gtile0, ng, blockIdx.x);
  int s = gsys[g];
  if (!pass_active(a, s, act)) return;
  const SysInfo &S = a.sys[s];
  const int K3 = L ? L : S.K[2], K3h = K3 / 2 + 1, nlines = S.K[0] * S.K[1];
  int tile = blockIdx.x - gtile0[g];
  int l0 = tile * 2 * FFT_PAIRS;
  int np = min(FFT_PAIRS, (nlines - l0) / 2);
  c2<T> *x = reinterpret_cast<c2<T> *>(smem_raw), *y = x + FFT_PAIRS * K3, *tws = y + FFT_PAIRS * K3;
  const c2<T> *C = a.C + S.cgrid0 + (size_t)l0 * K3h;
  for (int t = threadIdx.x; t < K3; t += blockDim.x) tws[t] = a.tw[S.tw[2] + t];
  staged_copy<FFT_PAIRS * L>(
      np * K3,
      [&](int t) {
        int cl = t / K3, m = t - cl * K3;
        int mm = m > K3 / 2 ? K3 - m : m;
        return c2pair<T>{C[(size_t)(2 * cl) * K3h + mm], C[(size_t)(2 * cl + 1) * K3h + mm]};
      },
      [&](int t, c2pair<T> p) {
        int cl = t / K3, m = t - cl * K3;
        bool up = m > K3 / 2;
        int mm = up ? K3 - m : m;
        c2<T> A = p.a, Bv = p.b;
        if (mm == 0 || 2 * mm == K3) { A.y = T(0); Bv.y = T(0); }
        if (up) { A.y = -A.y; Bv.y = -Bv.y; }
        c2<T> Z;
        Z.x = A.x - Bv.y; Z.y = A.y + Bv.x;
        x[cl * K3 + m] = Z;
      });
  __syncthreads();
  c2<T> *res = fft_lines<T, L>(x, y, K3, np, K3, S.rad[2], S.nst[2], tws, +1);
  T *Phi = a.Phi + S.rgrid0 + (size_t)l0 * K3;
  for (int t = threadIdx.x; t < 2 * np * K3; t += blockDim.x) {
    int rl = t / K3, k = t - rl * K3;
    c2<T> z = res[(rl >> 1) * K3 + k];
    Phi[t] = (rl & 1) ? z.y : z.x;
  }
}

// k2 pass (both directions): FFT_TILE consecutive columns (k1, m3) of the flattened K1 x K3h
// column index, each a line over k2 with stride K3h.
template <typename T, int L>
__global__ void __launch_bounds__(256) k_fft_y(Dev<T> a, const int *gsys, const int *gtile0, int ng, int act, int sign) {
  pdl_enter();
  extern __shared__ unsigned char smem_raw[];
  int g = group_member(gtile0, ng, blockIdx.x);
  int s = gsys[g];
  if (!pass_active(a, s, act)) return;
  const SysInfo &S = a.sys[s];
  const int K2 = L ? L : S.K[1], K3h = S.K3h, ncol = S.K[0] * K3h;
  int c0 = (blockIdx.x - gtile0[g]) * FFT_TILE;
  const int ld = K2 + 1;
  c2<T> *x = reinterpret_cast<c2<T> *>(smem_raw), *y = x + FFT_TILE * ld, *tws = y + FFT_TILE * ld;
  c2<T> *C = a.C + S.cgrid0;
  for (int t = threadIdx.x; t < K2; t += blockDim.x) tws[t] = a.tw[S.tw[1] + t];
  staged_copy<L * FFT_TILE>(
      K2 * FFT_TILE,
      [&](int t) {
        int k2 = t / FFT_TILE, c = t - k2 * FFT_TILE;
        int col = c0 + c;
        c2<T> v;
        v.x = T(0); v.y = T(0);
        if (col < ncol) {
          int k1 = col / K3h, m3 = col - k1 * K3h;
          v = C[((size_t)k1 * K2 + k2) * K3h + m3];
        }
        return v;
      },
      [&](int t, c2<T> v) {
        int k2 = t / FFT_TILE, c = t - k2 * FFT_TILE;
        x[c * ld + k2] = v;
      });
  __syncthreads();
  if (sign < 0) {
    // the real grid of this system was consumed by the k3 pass: clear this CTA's share of it for
    // the next spread (no separate memset between the sweeps)
    const size_t nq = (size_t)S.K[0] * S.K[1] * S.K[2];
    const int ntile = gtile0[g + 1] - gtile0[g];
    const size_t per = (nq + ntile - 1) / ntile, q0 = (size_t)(blockIdx.x - gtile0[g]) * per;
    const size_t q1 = q0 + per < nq ? q0 + per : nq;
    T *Qs = a.Q + S.rgrid0;
    for (size_t t = q0 + threadIdx.x; t < q1; t += blockDim.x) Qs[t] = T(0);
  }
  c2<T> *res = fft_lines<T, L, true>(x, y, K2, FFT_TILE, ld, S.rad[1], S.nst[1], tws, sign);
  for (int t = threadIdx.x; t < K2 * FFT_TILE; t += blockDim.x) {
    int k2 = t / FFT_TILE, c = t - k2 * FFT_TILE;
    int col = c0 + c;
    if (col < ncol) {
      int k1 = col / K3h, m3 = col - k1 * K3h;
      C[((size_t)k1 * K2 + k2) * K3h + m3] = res[c * ld + k2];
    }
  }
}

// ---- plane passes (meshes with K2 = K3 = L): one CTA per k1 plane runs the k3 and k2 passes in
// shared memory, in two regions of plane_region(L) complex elements each (the L/2 packed k3-lines
// of the real plane, or the L/2 + 1 k2-columns padded to L + 1).  The same arithmetic as
// k_fft_x_fwd followed by k_fft_y(-1), and as k_fft_y(+1) followed by k_fft_x_inv, with one grid
// round trip and one launch instead of two.
constexpr int PLANE_THREADS = 512;
__host__ __device__ constexpr int plane_region(int L) { return (L / 2 + 1) * (L + 1); }

template <typename T, int L>
__global__ void __launch_bounds__(PLANE_THREADS) k_fft_plane_fwd(Dev<T> a, const int *gsys, const int *gtile0, int ng, int act) {
  static_assert(L > 0 && L % 8 == 0, "compile-time plane length");
  pdl_enter();
  extern __shared__ unsigned char smem_raw[];
  const int g = group_member(gtile0, ng, blockIdx.x);
  const int s = gsys[g];
  if (!pass_active(a, s, act)) return;
  const SysInfo &S = a.sys[s];
  constexpr int K = L, Kh = L / 2 + 1, NP = L / 2, LD = L + 1, REG = plane_region(L), Q4 = L / 4;
  const int k1 = blockIdx.x - gtile0[g];
  c2<T> *A = reinterpret_cast<c2<T> *>(smem_raw), *B = A + REG, *tws = B + REG;
  for (int t = threadIdx.x; t < K; t += PLANE_THREADS) tws[t] = a.tw[S.tw[2] + t];  // K2 = K3: one table
  // rows 2cl and 2cl + 1 of the plane (K x K reals, rows k2) packed as complex line cl, four
  // columns per thread and load; each thread clears what it read (Q is zero for the next spread)
  using V = v4<T>;
  V *Qp = reinterpret_cast<V *>(a.Q + S.rgrid0 + (size_t)k1 * K * K);
  constexpr int NV = NP * Q4, PER = (NV + PLANE_THREADS - 1) / PLANE_THREADS;
  V lo[PER], hi[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int t = threadIdx.x + j * PLANE_THREADS;
    if (t < NV) {
      const int cl = t / Q4, q = t - cl * Q4;
      lo[j] = Qp[(2 * cl) * Q4 + q];
      hi[j] = Qp[(2 * cl + 1) * Q4 + q];
    }
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int t = threadIdx.x + j * PLANE_THREADS;
    if (t < NV) {
      const int cl = t / Q4, q = t - cl * Q4;
      c2<T> *d = A + cl * LD + 4 * q;  // line stride LD: odd in 8-byte words
      d[0].x = lo[j].x; d[0].y = hi[j].x;
      d[1].x = lo[j].y; d[1].y = hi[j].y;
      d[2].x = lo[j].z; d[2].y = hi[j].z;
      d[3].x = lo[j].w; d[3].y = hi[j].w;
      V z;
      z.x = T(0); z.y = T(0); z.z = T(0); z.w = T(0);
      Qp[(2 * cl) * Q4 + q] = z;
      Qp[(2 * cl + 1) * Q4 + q] = z;
    }
  }
  __syncthreads();
  c2<T> *res = fft_lines<T, L, true>(A, B, K, NP, LD, S.rad[2], S.nst[2], tws, -1);
  c2<T> *col = res == A ? B : A;
  // untangle line cl into rows 2cl, 2cl + 1 (m3 = 0..K/2), stored as k2-columns
  for (int t = threadIdx.x; t < NP * Kh; t += PLANE_THREADS) {
    const int cl = t / Kh, m = t - cl * Kh;
    const c2<T> Z = res[cl * LD + m], W = res[cl * LD + (m == 0 ? 0 : K - m)];
    c2<T> X0, X1;
    X0.x = T(0.5) * (Z.x + W.x); X0.y = T(0.5) * (Z.y - W.y);
    const T dx = Z.x - W.x, dy = Z.y + W.y;  // (Z - conj W) / (2 i)
    X1.x = T(0.5) * dy; X1.y = -T(0.5) * dx;
    col[m * LD + 2 * cl] = X0;
    col[m * LD + 2 * cl + 1] = X1;
  }
  __syncthreads();
  c2<T> *res2 = fft_lines<T, L, true>(col, res, K, Kh, LD, S.rad[1], S.nst[1], tws, -1);
  c2<T> *C = a.C + S.cgrid0 + (size_t)k1 * K * Kh;
  for (int t = threadIdx.x; t < K * Kh; t += PLANE_THREADS) {
    const int k2 = t / Kh, m3 = t - k2 * Kh;
    C[t] = res2[m3 * LD + k2];
  }
}

template <typename T, int L>
__global__ void __launch_bounds__(PLANE_THREADS) k_fft_plane_inv(Dev<T> a, const int *gsys, const int *gtile0, int ng, int act) {
  static_assert(L > 0 && L % 8 == 0, "compile-time plane length");
  pdl_enter();
  extern __shared__ unsigned char smem_raw[];
  const int g = group_member(gtile0, ng, blockIdx.x);
  const int s = gsys[g];
  if (!pass_active(a, s, act)) return;
  const SysInfo &S = a.sys[s];
  constexpr int K = L, Kh = L / 2 + 1, NP = L / 2, LD = L + 1, REG = plane_region(L), Q4 = L / 4;
  const int k1 = blockIdx.x - gtile0[g];
  c2<T> *A = reinterpret_cast<c2<T> *>(smem_raw), *B = A + REG, *tws = B + REG;
  for (int t = threadIdx.x; t < K; t += PLANE_THREADS) tws[t] = a.tw[S.tw[2] + t];
  const c2<T> *C = a.C + S.cgrid0 + (size_t)k1 * K * Kh;
  constexpr int NC = K * Kh, PER = (NC + PLANE_THREADS - 1) / PLANE_THREADS;
  c2<T> v[PER];
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int t = threadIdx.x + j * PLANE_THREADS;
    if (t < NC) v[j] = C[t];
  }
#pragma unroll
  for (int j = 0; j < PER; ++j) {
    const int t = threadIdx.x + j * PLANE_THREADS;
    if (t < NC) {
      const int k2 = t / Kh, m3 = t - k2 * Kh;
      A[m3 * LD + k2] = v[j];
    }
  }
  __syncthreads();
  c2<T> *res = fft_lines<T, L, true>(A, B, K, Kh, LD, S.rad[1], S.nst[1], tws, +1);
  c2<T> *lin = res == A ? B : A;
  // rows 2cl, 2cl + 1 back into complex line cl (z = a + i b) over the full k3 range (Hermitian)
  for (int t = threadIdx.x; t < NP * K; t += PLANE_THREADS) {
    const int cl = t / K, m = t - cl * K;
    const bool up = m > K / 2;
    const int mm = up ? K - m : m;
    c2<T> X0 = res[mm * LD + 2 * cl], X1 = res[mm * LD + 2 * cl + 1];
    if (mm == 0 || 2 * mm == K) { X0.y = T(0); X1.y = T(0); }
    if (up) { X0.y = -X0.y; X1.y = -X1.y; }
    c2<T> Z;
    Z.x = X0.x - X1.y; Z.y = X0.y + X1.x;
    lin[cl * LD + m] = Z;  // line stride LD: odd in 8-byte words
  }
  __syncthreads();
  c2<T> *res2 = fft_lines<T, L, true>(lin, res, K, NP, LD, S.rad[2], S.nst[2], tws, +1);
  using V = v4<T>;
  V *Pp = reinterpret_cast<V *>(a.Phi + S.rgrid0 + (size_t)k1 * K * K);
  for (int t = threadIdx.x; t < NP * Q4; t += PLANE_THREADS) {
    const int cl = t / Q4, q = t - cl * Q4;
    const c2<T> *z = res2 + cl * LD + 4 * q;
    V r0, r1;
    r0.x = z[0].x; r0.y = z[1].x; r0.z = z[2].x; r0.w = z[3].x;
    r1.x = z[0].y; r1.y = z[1].y; r1.z = z[2].y; r1.w = z[3].y;
    Pp[(2 * cl) * Q4 + q] = r0;
    Pp[(2 * cl + 1) * Q4 + q] = r1;
  }
}

// k1 pass with the convolution: FFT_TILE consecutive columns c = k2 K3h + m3 (contiguous in
// memory), forward FFT along k1, multiply by 2 G(m) (phi = dE/dQ = 2 K^3 irfft(G F[Q]),
// pme.py:370-376), inverse FFT.  With ENERGY the reciprocal energy sum w3 G |F|^2
// (pme.py:390-411) and the influence part of the virial are accumulated.
template <typename T, int L, bool ENERGY>
__global__ void __launch_bounds__(256) k_fft_z_conv(Dev<T> a, const int *gsys, const int *gtile0, int ng, int act) {
  pdl_enter();
  extern __shared__ unsigned char smem_raw[];
  __shared__ double red[7][8];
  int g = group_member(gtile0, ng, blockIdx.x);
  int s = gsys[g];
  if (!pass_active(a, s, act)) return;
  const SysInfo &S = a.sys[s];
  const int K1 = L ? L : S.K[0], K2 = S.K[1], K3 = S.K[2], K3h = S.K3h, ncol = K2 * K3h;
  int c0 = (blockIdx.x - gtile0[g]) * FFT_TILE;
  const int ld = K1 + 1;
  c2<T> *x = reinterpret_cast<c2<T> *>(smem_raw), *y = x + FFT_TILE * ld, *tws = y + FFT_TILE * ld;
  c2<T> *C = a.C + S.cgrid0;
  const size_t rs = (size_t)ncol;
  for (int t = threadIdx.x; t < K1; t += blockDim.x) tws[t] = a.tw[S.tw[0] + t];
  const T *G = a.Ginf + S.cgrid0;
  // the influence values of this tile are staged beside the grid columns (their loads in flight
  // with the grid's); y holds them until the first transform overwrites it
  T *gst = reinterpret_cast<T *>(y);
  staged_copy<L * FFT_TILE>(
      K1 * FFT_TILE,
      [&](int t) {
        int k1 = t / FFT_TILE, c = t - k1 * FFT_TILE;
        int col = c0 + c;
        c2pair<T> v;
        v.a.x = T(0); v.a.y = T(0); v.b.x = T(0); v.b.y = T(0);
        if (col < ncol) { v.a = C[k1 * rs + col]; v.b.x = G[k1 * rs + col]; }
        return v;
      },
      [&](int t, c2pair<T> v) {
        int k1 = t / FFT_TILE, c = t - k1 * FFT_TILE;
        x[c * ld + k1] = v.a;
        gst[t] = v.b.x;
      });
  __syncthreads();
  T gvr[(L * FFT_TILE + FFT_THREADS - 1) / FFT_THREADS > 0 ? (L * FFT_TILE + FFT_THREADS - 1) / FFT_THREADS : 1];
  if constexpr (L > 0) {
#pragma unroll
    for (int j = 0; j < (L * FFT_TILE + FFT_THREADS - 1) / FFT_THREADS; ++j) {
      int t = threadIdx.x + j * FFT_THREADS;
      gvr[j] = t < K1 * FFT_TILE ? gst[t] : T(0);
    }
    __syncthreads();  // y is the transform's scratch from here
  }
  c2<T> *res = fft_lines<T, L, true>(x, y, K1, FFT_TILE, ld, S.rad[0], S.nst[0], tws, -1);
  c2<T> *oth = res == x ? y : x;
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  const BoxInfo &B = a.box[s];
#pragma unroll
  for (int j = 0; j < (L > 0 ? (L * FFT_TILE + FFT_THREADS - 1) / FFT_THREADS : 1); ++j) {
   for (int t = threadIdx.x + j * FFT_THREADS; t < K1 * FFT_TILE; t += (L > 0 ? K1 * FFT_TILE : (int)blockDim.x)) {
    int k1 = t / FFT_TILE, c = t - k1 * FFT_TILE;
    int col = c0 + c;
    if (col >= ncol) continue;
    T gv = L > 0 ? gvr[j] : G[k1 * rs + col];
    c2<T> F = res[c * ld + k1];
    if (ENERGY && gv != T(0)) {
      int k2 = col / K3h, m3 = col - k2 * K3h;
      double w3 = (m3 == 0 || 2 * m3 == K3) ? 1.0 : 2.0;
      double e = w3 * double(gv) * (double(F.x) * double(F.x) + double(F.y) * double(F.y));
      int m1 = k1 <= (K1 - 1) / 2 ? k1 : k1 - K1;
      int m2 = k2 <= (K2 - 1) / 2 ? k2 : k2 - K2;
      if (K1 % 2 == 0 && k1 == K1 / 2) m1 = -K1 / 2;
      if (K2 % 2 == 0 && k2 == K2 / 2) m2 = -K2 / 2;
      double mv[3];
      for (int cc = 0; cc < 3; ++cc) mv[cc] = m1 * B.Hinv[cc * 3 + 0] + m2 * B.Hinv[cc * 3 + 1] + m3 * B.Hinv[cc * 3 + 2];
      double msq = mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2];
      double fac = 2.0 * (PI * PI / (a.beta * a.beta) + 1.0 / msq);
      acc[0] += e;
      acc[1] += e * (fac * mv[0] * mv[0] - 1.0);
      acc[2] += e * (fac * mv[1] * mv[1] - 1.0);
      acc[3] += e * (fac * mv[2] * mv[2] - 1.0);
      acc[4] += e * fac * mv[0] * mv[1];
      acc[5] += e * fac * mv[0] * mv[2];
      acc[6] += e * fac * mv[1] * mv[2];
    }
    T g2 = T(2) * gv;
    F.x *= g2; F.y *= g2;
    res[c * ld + k1] = F;
   }
  }
  if (ENERGY) {
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = 0; k < 7; ++k) {
      double v = warp_sum<double>(acc[k]);
      if (lane == 0) red[k][warp] = v;
    }
  }
  __syncthreads();
  if (ENERGY && threadIdx.x < 7) {
    double v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
    atomicAdd(&a.eacc[s].vinf[threadIdx.x], v);
  }
  c2<T> *res2 = fft_lines<T, L, true>(res, oth, K1, FFT_TILE, ld, S.rad[0], S.nst[0], tws, +1);
  for (int t = threadIdx.x; t < K1 * FFT_TILE; t += blockDim.x) {
    int k1 = t / FFT_TILE, c = t - k1 * FFT_TILE;
    int col = c0 + c;
    if (col < ncol) C[k1 * rs + col] = res2[c * ld + k1];
  }
}

// ------------------------------------------------------------------ row field + PME gather
// One warp (or group of LPA lanes) per atom.  s_i = sum_k de_ik/dd_i (forcefield.py:1395-1402) + dU_rec/dd_i
// (pme.py:378-388), then by MODE:
//   0 FIELD  out = -(s - c_self d)                       (forcefield.py:1428-1433)
//   1 OPER   out = d / alpha + s - c_self d, and p.Ap    (forcefield.py:1694-1712, 1806-1807)
// The row part alone: F_i = sum_k de_ik/dd_i (runs beside the PME chain).  LPR lanes per row
// (32: a warp per atom; 16 or 8: two or four atoms per warp, each row split over fewer lanes, more
// rows in flight per warp), 8 atoms per block of 8 LPR threads either way -- the autotuner's choice
// (Engine::autotune).  The lane partial sums are combined by a butterfly within each LPR group,
// so the variants differ only in the order of the row's additions.
template <typename T, bool WITH_Q, int ACT, int LPR = 32>
__global__ void __launch_bounds__(8 * LPR) k_rowfield(Dev<T> a, const v4<T> *__restrict__ D, v4<T> *__restrict__ F, int nvb) {
  static_assert(LPR == 32 || LPR == 16 || LPR == 8, "lanes per row");
  pdl_enter();
  const int sub = threadIdx.x / LPR, lane = threadIdx.x % LPR;
  // blocks of 8 rows (nvb of them); a grid smaller than nvb walks them at its stride (the row field
  // beside the FFT chain on a limited number of SMs)
  for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
  int s = a.wb_sys[vb];
  int i = a.wb_atom0[vb] + sub;
  const SysInfo &S = a.sys[s];
  if (ACT == 1 && !a.cg[s].active) continue;  // uniform over the block
  if (ACT == 2 && !a.cg[s].sweep2) continue;
  if (ACT == 3 && !a.cg[s].fallback) continue;
  const bool valid = i < S.atom0 + S.natom;
  if (LPR == 32 && !valid) continue;  // uniform over the warp
  int n = valid ? min(a.rn[i], a.mce) : 0;
  size_t base = (size_t)(valid ? i : 0) * a.mc;
  T f0 = 0, f1 = 0, f2 = 0;
  auto pair = [&](int k, T x, T y, T z, T g1, T g2) {
    v4<T> dk = D[k];
    T dkx = dk.x * x + dk.y * y + dk.z * z;
    T c = -g2 * dkx;
    if (WITH_Q) c -= a.q[k] * g1;
    f0 += c * x + g1 * dk.x;
    f1 += c * y + g1 * dk.y;
    f2 += c * z + g1 * dk.z;
  };
  if constexpr (sizeof(T) == 4) {
    const int4 *k4 = reinterpret_cast<const int4 *>(a.rk + base);
    const float4 *x4 = reinterpret_cast<const float4 *>(a.rx + base), *y4 = reinterpret_cast<const float4 *>(a.ry + base),
                 *z4 = reinterpret_cast<const float4 *>(a.rz + base), *p4 = reinterpret_cast<const float4 *>(a.rg1 + base),
                 *q4 = reinterpret_cast<const float4 *>(a.rg2 + base);
    // streaming loads (evict first): the 90+ MB of rows pass through L2 once per sweep and must
    // not push out the PME grids that the FFT passes read next.  The next group of four entries
    // is loaded before the current one is used (two groups of row data in flight per lane).
    int4 kk = make_int4(0, 0, 0, 0);
    float4 xx = make_float4(0, 0, 0, 0), yy = xx, zz = xx, g1 = xx, g2 = xx;
    if (4 * lane < n) {
      kk = __ldcs(k4 + lane);
      xx = __ldcs(x4 + lane); yy = __ldcs(y4 + lane); zz = __ldcs(z4 + lane); g1 = __ldcs(p4 + lane); g2 = __ldcs(q4 + lane);
    }
    for (int t4 = lane; 4 * t4 < n; t4 += LPR) {
      const int t4n = t4 + LPR;
      int4 kn = make_int4(0, 0, 0, 0);
      float4 xn = make_float4(0, 0, 0, 0), yn = xn, zn = xn, g1n = xn, g2n = xn;
      if (4 * t4n < n) {
        kn = __ldcs(k4 + t4n);
        xn = __ldcs(x4 + t4n); yn = __ldcs(y4 + t4n); zn = __ldcs(z4 + t4n); g1n = __ldcs(p4 + t4n); g2n = __ldcs(q4 + t4n);
      }
      int t = 4 * t4;
      pair(kk.x, xx.x, yy.x, zz.x, g1.x, g2.x);
      if (t + 1 < n) pair(kk.y, xx.y, yy.y, zz.y, g1.y, g2.y);
      if (t + 2 < n) pair(kk.z, xx.z, yy.z, zz.z, g1.z, g2.z);
      if (t + 3 < n) pair(kk.w, xx.w, yy.w, zz.w, g1.w, g2.w);
      kk = kn; xx = xn; yy = yn; zz = zn; g1 = g1n; g2 = g2n;
    }
  } else {
    for (int t = lane; t < n; t += LPR) {
      size_t o = base + t;
      pair(a.rk[o], a.rx[o], a.ry[o], a.rz[o], a.rg1[o], a.rg2[o]);
    }
  }
  // every lane of the warp takes part in the butterfly (a row past the system's end adds zeros)
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) {
    f0 += __shfl_xor_sync(0xffffffffu, f0, o);
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
  }
  if (valid && lane == 0) {
    v4<T> o;
    o.x = f0; o.y = f1; o.z = f2; o.w = T(0);
    F[i] = o;
  }
  }
}

// ROWS: the row sum is computed here; otherwise it is read from a.F (k_rowfield).  COMBINE (the
// CG direction's sweep with the row field started before the spread): a.F holds the rows of
// z, and the rows of p = z + beta p_prev are a.F + beta a.Fp (a.Fp: those of p_prev, rewritten).
template <typename T, int P, bool WITH_Q, int MODE, int ACT, bool ROWS = true, bool COMBINE = false, int LPA = 32>
__global__ void __launch_bounds__(8 * LPA) k_rowmat(Dev<T> a, const v4<T> *__restrict__ D, v4<T> *__restrict__ out) {
  static_assert(LPA == 32 || LPA == 16 || LPA == 8 || LPA == 4, "lanes per atom");
  pdl_enter();
  __shared__ T sh[WARPS_PER_BLOCK][2][3][P];  // per atom of the block
  __shared__ double red[WARPS_PER_BLOCK];
  const int warp = threadIdx.x / LPA, lane = threadIdx.x % LPA;  // the atom's group of LPA lanes
  const unsigned gm = group_mask<LPA>();
  int s = a.wb_sys[blockIdx.x];
  int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  bool valid = i < S.atom0 + S.natom;
  if (ACT == 1 && !a.cg[s].active) return;   // uniform over the block
  if (ACT == 2 && !a.cg[s].sweep2) return;
  if (ACT == 3 && !a.cg[s].fallback) return;
  double dotv = 0.0;
  if (valid) {
    int n = ROWS ? min(a.rn[i], a.mce) : 0;
    size_t base = (size_t)i * a.mc;
    T f0 = 0, f1 = 0, f2 = 0;
    auto pair = [&](int k, T x, T y, T z, T g1, T g2) {
      v4<T> dk = D[k];
      T dkx = dk.x * x + dk.y * y + dk.z * z;
      T c = -g2 * dkx;
      if (WITH_Q) c -= a.q[k] * g1;
      f0 += c * x + g1 * dk.x;
      f1 += c * y + g1 * dk.y;
      f2 += c * z + g1 * dk.z;
    };
    if constexpr (sizeof(T) == 4) {
      // 16-byte loads: each lane takes 4 consecutive entries of the row (capacity is a multiple of 32)
      const int4 *k4 = reinterpret_cast<const int4 *>(a.rk + base);
      const float4 *x4 = reinterpret_cast<const float4 *>(a.rx + base), *y4 = reinterpret_cast<const float4 *>(a.ry + base),
                   *z4 = reinterpret_cast<const float4 *>(a.rz + base), *p4 = reinterpret_cast<const float4 *>(a.rg1 + base),
                   *q4 = reinterpret_cast<const float4 *>(a.rg2 + base);
      for (int t4 = lane; 4 * t4 < n; t4 += LPA) {
        int4 kk = k4[t4];
        float4 xx = x4[t4], yy = y4[t4], zz = z4[t4], g1 = p4[t4], g2 = q4[t4];
        int t = 4 * t4;
        pair(kk.x, xx.x, yy.x, zz.x, g1.x, g2.x);
        if (t + 1 < n) pair(kk.y, xx.y, yy.y, zz.y, g1.y, g2.y);
        if (t + 2 < n) pair(kk.z, xx.z, yy.z, zz.z, g1.z, g2.z);
        if (t + 3 < n) pair(kk.w, xx.w, yy.w, zz.w, g1.w, g2.w);
      }
    } else {
      for (int t = lane; t < n; t += LPA) {
        size_t o = base + t;
        pair(a.rk[o], a.rx[o], a.ry[o], a.rz[o], a.rg1[o], a.rg2[o]);
      }
    }
    const BoxInfo &B = a.box[s];
    int4 b = a.base[i];
    v4<T> fr = a.frac[i];
    if (lane < 3) {
      T th[P], dth[P];
      bspline<T, P, false>(lane == 0 ? fr.x : (lane == 1 ? fr.y : fr.z), th, dth, nullptr);
#pragma unroll
      for (int k = 0; k < P; ++k) { sh[warp][0][lane][k] = th[k]; sh[warp][1][lane][k] = dth[k]; }
    }
    __syncwarp(gm);
    const T *phi = a.Phi + S.rgrid0;
    const int K1 = S.K[0], K2 = S.K[1], K3 = S.K[2];
    T g0 = 0, g1 = 0, g2 = 0;
    bool vec = false;
    if constexpr (sizeof(T) == 4) vec = (K3 & 3) == 0 && (S.rgrid0 & 3) == 0;
    if (vec) {
      // 16-byte loads: along k3 the P points of a stencil row fall into ng aligned groups of 4;
      // one work item per (stencil row, group)
      const int g0i = b.z >> 2, ng = ((b.z + P - 1) >> 2) - g0i + 1, K34 = K3 >> 2;
      for (int sl = lane; sl < P * P * ng; sl += LPA) {
        const int r = ng == 2 ? (sl >> 1) : (ng == 3 ? sl / 3 : sl / ng), gi = sl - r * ng;  // no runtime division for 2, 3
        const int j1 = r / P, j2 = r - j1 * P;
        int i1 = b.x + j1; if (i1 >= K1) i1 -= K1;
        int i2 = b.y + j2; if (i2 >= K2) i2 -= K2;
        const int g = g0i + gi, gp = g >= K34 ? g - K34 : g;
        const float4 ph4 = reinterpret_cast<const float4 *>(phi + ((size_t)i1 * K2 + i2) * K3)[gp];
        const T t1 = sh[warp][0][0][j1], t2 = sh[warp][0][1][j2];
        const T u1 = sh[warp][1][0][j1], u2 = sh[warp][1][1][j2];
        const T A0 = u1 * t2, A1 = t1 * u2, A2 = t1 * t2;
        const float pv[4] = {ph4.x, ph4.y, ph4.z, ph4.w};
#pragma unroll
        for (int el = 0; el < 4; ++el) {
          const int j3 = 4 * g + el - b.z;
          if (j3 >= 0 && j3 < P) {
            const T ph = T(pv[el]), t3 = sh[warp][0][2][j3], u3 = sh[warp][1][2][j3];
            g0 += ph * A0 * t3;
            g1 += ph * A1 * t3;
            g2 += ph * A2 * u3;
          }
        }
      }
    } else {
      for (int p = lane; p < P * P * P; p += LPA) {
        int j1 = p / (P * P), j2 = (p / P) % P, j3 = p % P;
        int i1 = b.x + j1; if (i1 >= K1) i1 -= K1;
        int i2 = b.y + j2; if (i2 >= K2) i2 -= K2;
        int i3 = b.z + j3; if (i3 >= K3) i3 -= K3;
        T ph = phi[((size_t)i1 * K2 + i2) * K3 + i3];
        T t1 = sh[warp][0][0][j1], t2 = sh[warp][0][1][j2], t3 = sh[warp][0][2][j3];
        T u1 = sh[warp][1][0][j1], u2 = sh[warp][1][1][j2], u3 = sh[warp][1][2][j3];
        g0 += ph * u1 * t2 * t3;
        g1 += ph * t1 * u2 * t3;
        g2 += ph * t1 * t2 * u3;
      }
    }
    if (ROWS) { f0 = group_sum<T, LPA>(f0, gm); f1 = group_sum<T, LPA>(f1, gm); f2 = group_sum<T, LPA>(f2, gm); }
    g0 = group_sum<T, LPA>(g0, gm); g1 = group_sum<T, LPA>(g1, gm); g2 = group_sum<T, LPA>(g2, gm);
    if (lane == 0) {
      if (!ROWS) { v4<T> fr = a.F[i]; f0 = fr.x; f1 = fr.y; f2 = fr.z; }
      if (COMBINE) {
        const double beta = a.cg[s].beta;
        if (beta != 0.0) {
          const v4<T> fp = a.Fp[i];
          f0 += T(beta) * fp.x; f1 += T(beta) * fp.y; f2 += T(beta) * fp.z;
        }
        a.Fp[i] = v4<T>{f0, f1, f2, T(0)};
      }
      // dU/dd_b = sum_a g_a Hinv[b][a] K_a
      T es[9];
#pragma unroll
      for (int bb = 0; bb < 3; ++bb)
#pragma unroll
        for (int aa = 0; aa < 3; ++aa) es[bb * 3 + aa] = T(B.Hinv[bb * 3 + aa] * S.K[aa]);
      T r0 = g0 * es[0] + g1 * es[1] + g2 * es[2];
      T r1 = g0 * es[3] + g1 * es[4] + g2 * es[5];
      T r2 = g0 * es[6] + g1 * es[7] + g2 * es[8];
      v4<T> di = D[i];
      T cs = T(a.c_self);
      v4<T> o;
      if (MODE == 0) {
        o.x = -(f0 + r0 - cs * di.x); o.y = -(f1 + r1 - cs * di.y); o.z = -(f2 + r2 - cs * di.z);
      } else {
        T ia = a.ialpha[i];
        o.x = di.x * ia + f0 + r0 - cs * di.x;
        o.y = di.y * ia + f1 + r1 - cs * di.y;
        o.z = di.z * ia + f2 + r2 - cs * di.z;
        dotv = double(di.x * o.x) + double(di.y * o.y) + double(di.z * o.z);
      }
      o.w = T(0);
      out[i] = o;
    }
  }
  if (MODE == 1) {
    if (lane == 0) red[warp] = dotv;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0;
      for (int w = 0; w < WARPS_PER_BLOCK; ++w) v += red[w];
      atomicAdd(&a.cg[s].acc_pap, v);
    }
  }
}

// ------------------------------------------------------------------ learned guess: features
// The model predicts the correction delta = mu* - x4 to the mu4 extrapolation x4 = 4 mu1 - 6 mu2 +
// 4 mu3 - mu4 (mu_j the converged dipoles j steps back), so the untrained model (zero output) is the
// reference's mu4 predictor, and the solver keeps its fused one-sweep start: everything the model
// sees is known before the step's first field sweep.
//
// Step 1, one warp per atom over its pair row, edges r < rg (the short-range graph): the permanent
// field of the graph, b_i = -sum_k [(-q_k G1 - G2 (p_k . x)) x + G1 p_k] (the real-space row field
// of charges and permanent dipoles, restricted to the graph), and three per-atom channel vectors
// (e nm): c0 = alpha_i (b_i - b_prev,i) (zero when there is no previous b), c1 = mu1 - mu2,
// c2 = x4 - mu1.  b overwrites b_prev (the same thread reads it first), for the next step.
// NN_CHAN floats per atom: c0, c1, c2 (3 each) and mu1 (3).
constexpr int NN_CHAN = 12;
// The graph edges of atom i from the list the row build wrote, one edge per lane and round (edges past
// nn_emax are not read, as in the message-passing model).
template <int LPA = 32, typename T, typename F>
__device__ __forceinline__ void for_graph_edges(const Dev<T> &a, int i, F &&edge) {
  const int lane = threadIdx.x % LPA;
  const int ne = min(a.nn_ne[i], a.nn_emax);
  const float4 *list = a.nn_e4 + (size_t)i * a.nn_emax;
  for (int e = lane; e < ne; e += LPA) {
    const float4 v = list[e];
    edge(__float_as_int(v.w), v.x, v.y, v.z, e);
  }
}

// Step 1, one warp per atom over the graph edges of its pair row (r < rg): the permanent field of
// the graph, b_i = -sum_k [(-q_k G1 - G2 (p_k . x)) x + G1 p_k] (the real-space row field of
// charges and permanent dipoles, restricted to the graph), and three per-atom channel vectors
// (e nm): c0 = alpha_i (b_i - b_prev,i) (zero when there is no previous b), c1 = mu1 - mu2,
// c2 = x4 - mu1.  b overwrites b_prev (the same thread reads it first), for the next step.
// NN_CHAN floats per atom: c0, c1, c2 (3 each) and mu1 (3).
template <typename T, int LPA = 32>
__global__ void __launch_bounds__(8 * LPA, 8 * 32 / LPA) k_nn_chan(Dev<T> a, const double *hist, const float4 *bl_prev,
                                                                  const int *valid, float rg, float4 *bl_out, float *chan) {
  static_assert(LPA == 32 || LPA == 16 || LPA == 8, "lanes per atom");
  const int warp = threadIdx.x / LPA, lane = threadIdx.x % LPA;  // the atom's group of LPA lanes
  const unsigned gm = group_mask<LPA>();
  int s = a.wb_sys[blockIdx.x];
  int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  if (i >= S.atom0 + S.natom) return;
  (void)rg;  // the graph radius is a.nn_rg2 here
  float f0 = 0.f, f1 = 0.f, f2 = 0.f;
  const float2 *G = a.nn_g + (size_t)i * a.nn_emax;
  for_graph_edges<LPA>(a, i, [&](int k, float x, float y, float z, int e) {
    const float2 g = G[e];  // the edge's pair kernels G1, G2, as the row build evaluated them
    const float g1 = g.x, g2 = g.y;
    double4 pk = a.pperm[k];
    float px = float(pk.x), py = float(pk.y), pz = float(pk.z);
    float c = -float(a.q[k]) * g1 - g2 * (px * x + py * y + pz * z);
    f0 += c * x + g1 * px;
    f1 += c * y + g1 * py;
    f2 += c * z + g1 * pz;
  });
  f0 = -group_sum<float, LPA>(f0, gm); f1 = -group_sum<float, LPA>(f1, gm); f2 = -group_sum<float, LPA>(f2, gm);
  if (lane >= 3) return;
  // lanes 0..2 write one component each
  const float fb = lane == 0 ? f0 : (lane == 1 ? f1 : f2);
  const float *bp = bl_prev ? reinterpret_cast<const float *>(bl_prev + i) : nullptr;
  const bool have_prev = bp && (!valid || *valid);
  const float db = have_prev ? fb - bp[lane] : 0.f;
  const size_t st = (size_t)a.nt * 3;
  double m1 = hist[3 * (size_t)i + lane], m2 = hist[st + 3 * (size_t)i + lane], m3 = hist[2 * st + 3 * (size_t)i + lane],
         m4 = hist[3 * st + 3 * (size_t)i + lane];
  double x4 = 4.0 * m1 - 6.0 * m2 + 4.0 * m3 - m4;
  reinterpret_cast<float *>(bl_out + i)[lane] = fb;
  if (lane == 0) reinterpret_cast<float *>(bl_out + i)[3] = 0.f;
  float *C = chan + (size_t)i * NN_CHAN;
  C[lane] = float(a.alpha[i]) * db;
  C[3 + lane] = float(m1 - m2);
  C[6 + lane] = float(x4 - m1);
  C[9 + lane] = float(m1);
}

// Step 2, one warp per atom over the same edges: vector channels (NN_CH = 15) v0..v2 = the atom's own
// c0..c2 and, for each c and 2 radial bases phi_k(r) = exp(-((r - (0.15 + 0.2 k) nm) / 0.15 nm)^2)
// (cos(pi r / rg) + 1) / 2, the aggregates A_ck = sum_j phi_k c_j and D_ck = sum_j phi_k (c_j . u) u
// (u = x / r), 36 sums in one pass over the edges with a transposing warp reduction; 16 rotation
// invariants (asinh of magnitudes and dot products over the change scale sigma, |mu1| over
// 0.02 e nm, alpha, radius).  The model mixes the 15 channels, so the predicted correction turns
// with the system.  Sets *valid (the next step has a previous b).
// One halving step of a transposing warp reduction: lanes with bit (N/2) set keep the upper half of
// their N values and receive the partner's upper half, the others the lower halves.
template <int N>
__device__ __forceinline__ void transpose_step(float (&v)[32], int lane) {
  const bool up = lane & (N / 2);
#pragma unroll
  for (int j = 0; j < N / 2; ++j) {
    float send = up ? v[j] : v[j + N / 2];
    float keep = up ? v[j + N / 2] : v[j];
    v[j] = keep + __shfl_xor_sync(0xffffffffu, send, N / 2);
  }
}
// Warp sums of 32 values per lane in 31 shuffles: lane l returns the total of v[l].
__device__ __forceinline__ float warp_transpose_sum(float (&v)[32]) {
  const int lane = threadIdx.x & 31;
  transpose_step<32>(v, lane);
  transpose_step<16>(v, lane);
  transpose_step<8>(v, lane);
  transpose_step<4>(v, lane);
  transpose_step<2>(v, lane);
  return v[0];
}

// The 36 sums over the graph edges in one pass, value o = ((q * 3 + c) * 2 + k) * 3 + x for the
// plain (q = 0: A) and projected (q = 1: D) sums of channel c with radial basis k; returns on lane l
// the total of value l (l < 32) and in tail[0..3] the totals of values 32..35.
template <typename T>
__device__ __forceinline__ float nn_aggregate(const Dev<T> &a, int i, const float *chan, float rg, float (&tail)[4]) {
  float acc[36];
#pragma unroll
  for (int o = 0; o < 36; ++o) acc[o] = 0.f;
  const float irg = 1.f / rg;
  for_graph_edges(a, i, [&](int j, float x, float y, float z, int) {
    float r = sqrtf(x * x + y * y + z * z);
    float ir = 1.f / r, u[3] = {x * ir, y * ir, z * ir};
    float fc = 0.5f * (cospif(r * irg) + 1.f);
    float phi[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      float d = (r - (0.15f + 0.2f * k)) * (1.f / 0.15f);
      phi[k] = expf(-d * d) * fc;
    }
    const float4 *cj = reinterpret_cast<const float4 *>(chan + (size_t)j * NN_CHAN);
    float4 c01 = cj[0], c12 = cj[1], c2m = cj[2];
    float v[3][3] = {{c01.x, c01.y, c01.z}, {c01.w, c12.x, c12.y}, {c12.z, c12.w, c2m.x}};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float pr = v[c][0] * u[0] + v[c][1] * u[1] + v[c][2] * u[2];
#pragma unroll
      for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int xx = 0; xx < 3; ++xx) {
          acc[(c * 2 + k) * 3 + xx] += phi[k] * v[c][xx];
          acc[18 + (c * 2 + k) * 3 + xx] += phi[k] * pr * u[xx];
        }
    }
  });
#pragma unroll
  for (int o = 0; o < 4; ++o) tail[o] = warp_sum<float>(acc[32 + o]);
  float (&head)[32] = *reinterpret_cast<float (*)[32]>(acc);
  return warp_transpose_sum(head);
}

template <typename T>
__global__ void __launch_bounds__(256, 4) k_nn_features(Dev<T> a, const float *chan, float sigma, float rg, float *inv, float *vec,
                                                     int *valid) {
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (valid && blockIdx.x == 0 && threadIdx.x == 0) *valid = 1;  // read by the previous kernel only
  int s = a.wb_sys[blockIdx.x];
  int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  if (i >= S.atom0 + S.natom) return;
  float *V = vec + (size_t)i * pgmnn::NN_CH * 3;
  float *F = inv + (size_t)i * pgmnn::NN_IN;
  const float is = 1.f / sigma, is2 = is * is;
  float tail[4];
  // lane l holds value l; the norms of the first eight (c, k) groups of three for the invariants
  float mine = nn_aggregate(a, i, chan, rg, tail);
  V[9 + lane] = mine;
  if (lane < 4) V[9 + 32 + lane] = tail[lane];
  float sq = mine * mine;
  float n2 = sq + __shfl_down_sync(0xffffffffu, sq, 1) + __shfl_down_sync(0xffffffffu, sq, 2);
  // the 16 invariants on 16 lanes at once: F[8 + l / 3] on lanes l = 0, 3, .., 21 (the group norms),
  // F[l - 24] on lanes 24..31 (the atom's own channels, |mu1|, alpha, radius); V[0..8] the own channels
  const float *ci = chan + (size_t)i * NN_CHAN;
  if (lane < 9) V[lane] = ci[lane];
  float arg = 0.f;
  bool ash = true;
  int slot = -1;
  if (lane < 24) {
    if (lane % 3 == 0) { arg = sqrtf(n2) * is; slot = 8 + lane / 3; }
  } else {
    const float s0[3] = {ci[0], ci[1], ci[2]}, s1[3] = {ci[3], ci[4], ci[5]}, s2[3] = {ci[6], ci[7], ci[8]};
    const float m1[3] = {ci[9], ci[10], ci[11]};
    auto dot = [](const float *p, const float *q) { return p[0] * q[0] + p[1] * q[1] + p[2] * q[2]; };
    auto norm3 = [](const float *p) { return sqrtf(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]); };
    slot = lane - 24;
    switch (slot) {
      case 0: arg = float(a.alpha[i]) * 1e3f; ash = false; break;
      case 1: arg = float(a.radius[i]) / 0.06f; ash = false; break;
      case 2: arg = norm3(s0) * is; break;
      case 3: arg = norm3(m1) * 50.f; ash = false; break;
      case 4: arg = norm3(s1) * is; break;
      case 5: arg = norm3(s2) * is; break;
      case 6: arg = dot(s0, s1) * is2; break;
      default: arg = dot(s0, s2) * is2; break;
    }
  }
  if (slot >= 0) F[slot] = ash ? asinhf(arg) : arg;
}

template <typename T>
__global__ void k_copy_vec(int n, const v4<T> *src, v4<T> *dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i];
}

template <typename T>
__global__ void k_vec_from_f64(int n, const double *src, v4<T> *dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  v4<T> d;
  d.x = T(src[3 * i]); d.y = T(src[3 * i + 1]); d.z = T(src[3 * i + 2]); d.w = T(0);
  dst[i] = d;
}

// ------------------------------------------------------------------ CG
// Start, step 1 (thread per atom): the predictor guess x0h = sum c_j hist_j (forcefield.py:605,
// 1956-1958) and the dipoles of the first field sweep: p + x0h (fused start) or p (plain).
template <typename T>
__global__ void k_start1(Dev<T> a, const double *hist, int K, double c0, double c1, double c2, double c3, const float *xnn) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  int s = a.sysid[i];
  const CGSys &G = a.cg[s];
  double x0[3] = {0, 0, 0};
  if (G.have) {
    const double cc[4] = {c0, c1, c2, c3};
    for (int j = 0; j < K; ++j)
      for (int c = 0; c < 3; ++c) x0[c] += cc[j] * hist[((size_t)j * a.nt + i) * 3 + c];
    if (xnn)  // the learned correction to the extrapolation
      for (int c = 0; c < 3; ++c) x0[c] += double(xnn[3 * (size_t)i + c]);
  }
  double4 p = a.pperm[i];
  v4<T> d, x;
  if (G.fused) { d.x = T(p.x + x0[0]); d.y = T(p.y + x0[1]); d.z = T(p.z + x0[2]); }
  else { d.x = T(p.x); d.y = T(p.y); d.z = T(p.z); }
  d.w = T(0);
  x.x = T(x0[0]); x.y = T(x0[1]); x.z = T(x0[2]); x.w = T(0);
  a.D[i] = d;
  a.X[i] = x;
}

// Start, step 2: fused: r0 = field(q, p + x0) - x0 / alpha; plain: b = field(q, p), the norm
// mean|alpha b| and, without history, x0 = alpha b (forcefield.py:1960-1997).
template <typename T>
__global__ void k_start2(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  __shared__ double red[THREADS_PER_BLOCK / 32];
  int s = a.tb_sys[blockIdx.x];
  int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
  const SysInfo &S = a.sys[s];
  CGSys &G = a.cg[s];
  double sab = 0.0;
  if (i < S.atom0 + S.natom) {
    v4<T> b = a.B[i];
    v4<T> x = a.X[i];
    T al = a.alpha[i];
    if (G.fused) {
      T ia = a.ialpha[i];
      v4<T> r;
      r.x = b.x - x.x * ia; r.y = b.y - x.y * ia; r.z = b.z - x.z * ia; r.w = T(0);
      a.R[i] = r;
    } else {
      double ax = double(a.alpha[i]) * double(b.x), ay = double(a.alpha[i]) * double(b.y), az = double(a.alpha[i]) * double(b.z);
      sab = fabs(ax) + fabs(ay) + fabs(az);
      if (!G.have) { x.x = T(ax); x.y = T(ay); x.z = T(az); x.w = T(0); a.X[i] = x; }
      (void)al;
    }
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  sab = warp_sum<double>(sab);
  if (lane == 0) red[warp] = sab;
  __syncthreads();
  if (threadIdx.x == 0 && !G.fused) {
    double v = 0;
    for (int w = 0; w < THREADS_PER_BLOCK / 32; ++w) v += red[w];
    atomicAdd(&G.acc_abs, v);
  }
}

// Start, step 3 (plain start only): r0 = b - A x0.
template <typename T>
__global__ void k_start3(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  int s = a.sysid[i];
  if (a.cg[s].fused) return;
  v4<T> b = a.B[i], ap = a.AP[i], r;
  r.x = b.x - ap.x; r.y = b.y - ap.y; r.z = b.z - ap.z; r.w = T(0);
  a.R[i] = r;
}

// CG initialisation: z = alpha r, p = z, r.z and max|alpha r| (forcefield.py:1796-1819).
// FB (the learned guess's fallback, systems with the flag only): first back to the extrapolation,
// x = x4 = x - delta and r0 = b - A x4 = r0 + A delta (A delta in AP).
// LOCAL (the local preconditioner): only max|alpha r|; z, p and r.z come from its kernels.
template <typename T, bool FB = false, bool LOCAL = false>
__global__ void k_cg_init(Dev<T> a, const float *delta = nullptr) {
  __shared__ double red[THREADS_PER_BLOCK / 32];
  __shared__ unsigned long long mx[THREADS_PER_BLOCK / 32];
  if (FB) pdl_enter();  // launched as a programmatic dependent of the fallback sweep
  int s = a.tb_sys[blockIdx.x];
  if (FB && !a.cg[s].fallback) return;  // uniform over the block
  int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
  const SysInfo &S = a.sys[s];
  double rz = 0, m = 0;
  if (i < S.atom0 + S.natom) {
    if (FB) {
      v4<T> r = a.R[i], ad = a.AP[i], x = a.X[i];
      r.x += ad.x; r.y += ad.y; r.z += ad.z;
      x.x -= T(delta[3 * (size_t)i]); x.y -= T(delta[3 * (size_t)i + 1]); x.z -= T(delta[3 * (size_t)i + 2]);
      a.R[i] = r;
      a.X[i] = x;
    }
    v4<T> r = a.R[i];
    T al = a.alpha[i];
    v4<T> z;
    z.x = al * r.x; z.y = al * r.y; z.z = al * r.z; z.w = T(0);
    if (!LOCAL) {
      a.Z[i] = z;
      a.P[i] = z;
      rz = double(r.x * z.x) + double(r.y * z.y) + double(r.z * z.z);
    }
    m = fmax(fabs(double(z.x)), fmax(fabs(double(z.y)), fabs(double(z.z))));
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  rz = warp_sum<double>(rz);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) { red[warp] = rz; mx[warp] = (unsigned long long)__double_as_longlong(m); }
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    unsigned long long mm = 0;
    for (int w = 0; w < THREADS_PER_BLOCK / 32; ++w) { v += red[w]; mm = max(mm, mx[w]); }
    atomicAdd(&a.cg[s].acc_rz, v);
    atomicMax(&a.cg[s].acc_max, mm);
  }
}

// Per-system scalars after the start: norm, r.z, err, active; *any = some system iterates.
// The learned guess's check (fb_factor > 0, pass 0): a system that started from x4 + the model's
// correction falls back to x4 when its start residual err exceeds fb_factor times the running
// mean of the extrapolation's (raising the fallback node's condition, *fb_any); a system that
// started from the extrapolation itself adds its err to that mean.  Pass 1 (after the fallback
// sweep) re-evaluates the fallback systems, adds their (extrapolation) err to the mean and counts
// the fallback; *any covers every system.
__global__ void k_cg_begin(CGSys *cg, int nsys, double tol, int max_iter, int *any, double fb_factor = 0.0, int pass = 0,
                           cudaGraphConditionalHandle fbcond = 0, int use_cond = 0, int *fb_any = nullptr) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  __shared__ int act, fb;
  if (threadIdx.x == 0) { act = 0; fb = 0; }
  __syncthreads();
  constexpr double W = 0.1;  // weight of a new sample in the running mean
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    CGSys &G = cg[s];
    if (pass == 0 || G.fallback) {
      if (!G.fused) G.norm = G.acc_abs / G.n3 + 1e-300;
      G.rz = G.acc_rz;
      G.err = __longlong_as_double((long long)G.acc_max) / G.norm;
      G.beta = 0.0;
      G.it = 0;
      G.active = (G.err > (G.tol_s >= 0.0 ? G.tol_s : tol)) && ((G.maxit_s >= 0 ? G.maxit_s : max_iter) > 0);
      G.acc_abs = 0; G.acc_rz = 0; G.acc_max = 0; G.acc_pap = 0; G.acc_num = 0;
      const bool record = (pass == 1) || (fb_factor > 0.0 && G.have && !G.nn);
      if (pass == 0 && fb_factor > 0.0 && G.nn && G.ref_n > 0 && G.err > fb_factor * G.ref_err) {
        G.fallback = 1;
        atomicOr(&fb, 1);
      } else if (record) {
        G.ref_err = G.ref_n == 0 ? G.err : (1.0 - W) * G.ref_err + W * G.err;
        G.ref_n += 1;
        if (pass == 1) G.fallbacks += 1;
      }
    }
    if (G.active) atomicOr(&act, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *any = act;
    if (pass == 0 && fb_any) *fb_any = fb;
    if (pass == 0 && use_cond && fb) cudaGraphSetConditional(fbcond, 1u);  // the fallback node runs (default 0)
  }
}

// Fallback, step 1: the model's correction delta of every fallback system's atoms as the dipoles
// of one operator sweep (A delta).
template <typename T>
__global__ void k_fb_prep(Dev<T> a, const float *delta) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt || !a.cg[a.sysid[i]].fallback) return;
  v4<T> d;
  d.x = T(delta[3 * (size_t)i]); d.y = T(delta[3 * (size_t)i + 1]); d.z = T(delta[3 * (size_t)i + 2]); d.w = T(0);
  a.D[i] = d;
}

// One CG update (thread per atom): x += a p, r' = r - a Ap, z' = alpha r', and the sums of
// z'.(r' - r), r'.z', max|z'| (forcefield.py:1802-1814).
// One CG update (thread per atom): x += st p, r -= st Ap, z = alpha r (Jacobi), with the block
// partials of z.(r_new - r), r.z and max|z| added to the system's accumulators.
template <typename T>
__device__ __forceinline__ void cg_update_body(Dev<T> &a) {
  __shared__ double red[2][THREADS_PER_BLOCK / 32];
  __shared__ unsigned long long mx[THREADS_PER_BLOCK / 32];
  int s = a.tb_sys[blockIdx.x];
  CGSys &G = a.cg[s];
  if (!G.active) return;  // the block's system has converged
  int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
  const SysInfo &S = a.sys[s];
  double num = 0, rzn = 0, m = 0;
  if (i < S.atom0 + S.natom) {
    T st = T(G.rz / fmax(G.acc_pap, 1e-300));
    v4<T> x = a.X[i], r = a.R[i], p = a.P[i], ap = a.AP[i];
    T al = a.alpha[i];
    x.x += st * p.x; x.y += st * p.y; x.z += st * p.z;
    v4<T> rn, z;
    rn.x = r.x - st * ap.x; rn.y = r.y - st * ap.y; rn.z = r.z - st * ap.z; rn.w = T(0);
    z.x = al * rn.x; z.y = al * rn.y; z.z = al * rn.z; z.w = T(0);
    num = double(z.x * (rn.x - r.x)) + double(z.y * (rn.y - r.y)) + double(z.z * (rn.z - r.z));
    rzn = double(rn.x * z.x) + double(rn.y * z.y) + double(rn.z * z.z);
    m = fmax(fabs(double(z.x)), fmax(fabs(double(z.y)), fabs(double(z.z))));
    a.X[i] = x;
    a.R[i] = rn;
    a.Z[i] = z;
  }
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  num = warp_sum<double>(num);
  rzn = warp_sum<double>(rzn);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) { red[0][warp] = num; red[1][warp] = rzn; mx[warp] = (unsigned long long)__double_as_longlong(m); }
  __syncthreads();
  if (threadIdx.x == 0) {
    double v0 = 0, v1 = 0;
    unsigned long long mm = 0;
    for (int w = 0; w < THREADS_PER_BLOCK / 32; ++w) { v0 += red[0][w]; v1 += red[1][w]; mm = max(mm, mx[w]); }
    atomicAdd(&G.acc_num, v0);
    atomicAdd(&G.acc_rz, v1);
    atomicMax(&G.acc_max, mm);
  }
}

// The per-system scalars after an update (run by the last block of k_cg_update_check).
__device__ __forceinline__ void cg_check_body(CGSys *cg, int nsys, double tol, int max_iter, int *any,
                                              cudaGraphConditionalHandle cond, int use_cond) {
  __shared__ int act;
  if (threadIdx.x == 0) act = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    CGSys &G = cg[s];
    if (G.active) {
      G.beta = G.acc_num / fmax(G.rz, 1e-300);
      G.rz = G.acc_rz;
      G.err = __longlong_as_double((long long)G.acc_max) / G.norm;
      G.it += 1;
      G.active = (G.err > (G.tol_s >= 0.0 ? G.tol_s : tol)) && (G.it < (G.maxit_s >= 0 ? G.maxit_s : max_iter));
    }
    G.acc_num = 0; G.acc_rz = 0; G.acc_max = 0; G.acc_pap = 0;
    if (G.active) atomicOr(&act, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *any = act;
    if (use_cond) cudaGraphSetConditional(cond, act ? 1u : 0u);  // the captured while loop of the solve
  }
}

// The CG update and the per-system check in one launch: every block adds its partial sums, and the block that
// finishes last (a counter after a memory fence) evaluates the per-system scalars and the loop
// condition, then resets the counter for the next iteration.
template <typename T>
__global__ void k_cg_update_check(Dev<T> a, int nsys, double tol, int max_iter, int *any, cudaGraphConditionalHandle cond,
                                  int use_cond, unsigned *done) {
  pdl_enter();
  cg_update_body(a);
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this block's partial sums are visible before it is counted
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  cg_check_body(a.cg, nsys, tol, max_iter, any, cond, use_cond);
  if (threadIdx.x == 0) *done = 0u;
}

// ------------------------------------------------------------------ local preconditioner
// z = M^-1 r with local_niter > 0 inner CG iterations on A_loc v = v / alpha + sum over the row
// entries closer than local_cut of T v_k, T v = -G2 (v . x) x + G1 v (the row field's pair term),
// started from z = alpha r (forcefield.py:1766-1792; the outer CG is then flexible, with the
// Polak-Ribiere beta it already uses).  Thread per atom; the short entries compacted entry-major.

// sum over atom i's short entries of T v_k (get(k) = v_k)
template <typename T, typename Get>
__device__ __forceinline__ void short_sum(const Dev<T> &a, int i, Get &&get, T &f0, T &f1, T &f2) {
  const int n = a.sh_n[i];
#pragma unroll 4
  for (int e = 0; e < n; ++e) {
    const size_t c = (size_t)e * a.nt + i;
    const T x = a.c_x[c], y = a.c_y[c], z = a.c_z[c], g1 = a.c_g1[c], g2 = a.c_g2[c];
    const v4<T> v = get(a.c_k[c]);
    const T cc = -g2 * (v.x * x + v.y * y + v.z * z);
    f0 += cc * x + g1 * v.x;
    f1 += cc * y + g1 * v.y;
    f2 += cc * z + g1 * v.z;
  }
}

// the block's sum of v added to *dst (one atomic per block)
__device__ __forceinline__ void block_add(double v, double *dst) {
  __shared__ double red[THREADS_PER_BLOCK / 32];
  v = warp_sum<double>(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < THREADS_PER_BLOCK / 32; ++w) t += red[w];
    atomicAdd(dst, t);
  }
}

// Which systems a chain kernel serves: 0 all, 1 the iterating ones, 3 those falling back.
__device__ __forceinline__ bool lp_skip(int act, const CGSys &G) {
  return (act == 1 && !G.active) || (act == 3 && !G.fallback);
}

// Inner start: z = alpha r, rr = r - A_loc(alpha r) = -sum T (alpha r)_k, zz = alpha rr (the first
// inner direction), partial rr . zz.
template <typename T, int ACT>
__global__ void k_lp_start(Dev<T> a) {
  pdl_enter();
  const int s = a.tb_sys[blockIdx.x];
  CGSys &G = a.cg[s];
  if (lp_skip(ACT, G)) return;  // uniform over the block
  const int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
  const SysInfo &S = a.sys[s];
  double rz = 0.0;
  if (i < S.atom0 + S.natom) {
    T f0 = 0, f1 = 0, f2 = 0;
    short_sum(a, i, [&](int k) {
      const v4<T> r = a.R[k];
      const T al = a.alpha[k];
      v4<T> w;
      w.x = al * r.x; w.y = al * r.y; w.z = al * r.z; w.w = T(0);
      return w;
    }, f0, f1, f2);
    const v4<T> r = a.R[i];
    const T al = a.alpha[i];
    v4<T> z, rr, zz;
    z.x = al * r.x; z.y = al * r.y; z.z = al * r.z; z.w = T(0);
    rr.x = -f0; rr.y = -f1; rr.z = -f2; rr.w = T(0);
    zz.x = al * rr.x; zz.y = al * rr.y; zz.z = al * rr.z; zz.w = T(0);
    a.Z[i] = z;
    a.LRR[i] = rr;
    a.LZZ[i] = zz;
    a.LP0[i] = zz;  // the first inner direction (kept: the next direction adds to it)
    rz = double(rr.x * zz.x) + double(rr.y * zz.y) + double(rr.z * zz.z);
  }
  block_add(rz, &G.acc_lrz);
}

// Inner direction and its product: p = zz (FIRST) or zz + lb p_prev (written to Pout), Ap =
// A_loc(p) into AP (the neighbours' p formed the same way), partial p . Ap.
template <typename T, int ACT, bool FIRST>
__global__ void k_lp_ap(Dev<T> a, const v4<T> *__restrict__ Pin, v4<T> *__restrict__ Pout) {
  pdl_enter();
  const int s = a.tb_sys[blockIdx.x];
  CGSys &G = a.cg[s];
  if (lp_skip(ACT, G)) return;
  const int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
  const SysInfo &S = a.sys[s];
  const T b = T(G.lb);
  auto pget = [&](int k) {
    v4<T> p = a.LZZ[k];
    if (!FIRST) {
      const v4<T> q = Pin[k];
      p.x += b * q.x; p.y += b * q.y; p.z += b * q.z;
    }
    return p;
  };
  double pap = 0.0;
  if (i < S.atom0 + S.natom) {
    T f0 = 0, f1 = 0, f2 = 0;
    short_sum(a, i, pget, f0, f1, f2);
    const v4<T> p = pget(i);
    const T ia = a.ialpha[i];
    v4<T> ap;
    ap.x = p.x * ia + f0; ap.y = p.y * ia + f1; ap.z = p.z * ia + f2; ap.w = T(0);
    if (!FIRST) Pout[i] = p;
    a.AP[i] = ap;
    pap = double(p.x * ap.x) + double(p.y * ap.y) + double(p.z * ap.z);
  }
  block_add(pap, &G.acc_lpap);
}

// Inner update: z += al p (al = rr.zz / p.Ap); not LAST: rr -= al Ap, zz = alpha rr, partial rr.zz
// for the next inner iteration.  LAST: the outer quantities -- MODE 0 (start, fallback): p = z
// and r.z; MODE 1 (iteration): z.(r_new - r_old) and r_new.z.  The block that finishes last
// evaluates the inner scalars (lb, the next rr.zz) and, in MODE 1, the outer CG's per-system check
// and loop condition (cg_check_body).
template <typename T, int ACT, bool LAST, int MODE>
__global__ void k_lp_step(Dev<T> a, const v4<T> *__restrict__ Pcur, int nsys, double tol, int max_iter, int *any,
                          cudaGraphConditionalHandle cond, int use_cond, unsigned *done) {
  pdl_enter();
  {
    const int s = a.tb_sys[blockIdx.x];
    CGSys &G = a.cg[s];
    if (!lp_skip(ACT, G)) {
      const int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
      const SysInfo &S = a.sys[s];
      const T al = T(G.acc_lrz / fmax(G.acc_lpap, 1e-300));
      double v0 = 0.0, v1 = 0.0;
      if (i < S.atom0 + S.natom) {
        const v4<T> p = Pcur[i];
        v4<T> z = a.Z[i];
        z.x += al * p.x; z.y += al * p.y; z.z += al * p.z;
        a.Z[i] = z;
        if (!LAST) {
          const v4<T> ap = a.AP[i];
          v4<T> rr = a.LRR[i], zz;
          const T alpha = a.alpha[i];
          rr.x -= al * ap.x; rr.y -= al * ap.y; rr.z -= al * ap.z;
          zz.x = alpha * rr.x; zz.y = alpha * rr.y; zz.z = alpha * rr.z; zz.w = T(0);
          a.LRR[i] = rr;
          a.LZZ[i] = zz;
          v0 = double(rr.x * zz.x) + double(rr.y * zz.y) + double(rr.z * zz.z);
        } else if (MODE == 0) {
          const v4<T> r = a.R[i];
          a.P[i] = z;
          v0 = double(r.x * z.x) + double(r.y * z.y) + double(r.z * z.z);
        } else {
          const v4<T> r = a.R[i], dr = a.DR[i];
          v0 = double(z.x * dr.x) + double(z.y * dr.y) + double(z.z * dr.z);
          v1 = double(r.x * z.x) + double(r.y * z.y) + double(r.z * z.z);
        }
      }
      if (!LAST) {
        block_add(v0, &G.acc_lrz2);
      } else if (MODE == 0) {
        block_add(v0, &G.acc_rz);
      } else {
        block_add(v0, &G.acc_num);
        __syncthreads();
        block_add(v1, &G.acc_rz);
      }
    }
  }
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // this block's partial sums are visible before it is counted
    last = atomicAdd(done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    CGSys &G = a.cg[s];
    if (!LAST) {
      G.lb = G.acc_lrz2 / fmax(G.acc_lrz, 1e-300);
      G.acc_lrz = G.acc_lrz2;
    } else {
      G.acc_lrz = 0.0;
    }
    G.acc_lrz2 = 0.0;
    G.acc_lpap = 0.0;
  }
  if (LAST && MODE == 1) {
    __syncthreads();
    cg_check_body(a.cg, nsys, tol, max_iter, any, cond, use_cond);
  }
  if (threadIdx.x == 0) *done = 0u;
}

// The outer CG update with the local preconditioner (thread per atom): x += st p, r_new = r - st
// Ap, DR = r_new - r, and max|alpha r_new| (the convergence test stays pmemd-pgm's); z, r.z and
// the check follow in the preconditioner's kernels.
template <typename T>
__global__ void k_cg_update_r(Dev<T> a) {
  pdl_enter();
  __shared__ unsigned long long mx[THREADS_PER_BLOCK / 32];
  const int s = a.tb_sys[blockIdx.x];
  CGSys &G = a.cg[s];
  if (!G.active) return;  // uniform over the block
  const int i = a.tb_atom0[blockIdx.x] + threadIdx.x;
  const SysInfo &S = a.sys[s];
  double m = 0.0;
  if (i < S.atom0 + S.natom) {
    const T st = T(G.rz / fmax(G.acc_pap, 1e-300));
    v4<T> x = a.X[i], r = a.R[i];
    const v4<T> p = a.P[i], ap = a.AP[i];
    const T al = a.alpha[i];
    x.x += st * p.x; x.y += st * p.y; x.z += st * p.z;
    v4<T> rn, dr;
    rn.x = r.x - st * ap.x; rn.y = r.y - st * ap.y; rn.z = r.z - st * ap.z; rn.w = T(0);
    dr.x = rn.x - r.x; dr.y = rn.y - r.y; dr.z = rn.z - r.z; dr.w = T(0);
    a.X[i] = x;
    a.R[i] = rn;
    a.DR[i] = dr;
    m = fmax(fabs(double(al * rn.x)), fmax(fabs(double(al * rn.y)), fabs(double(al * rn.z))));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) mx[threadIdx.x >> 5] = (unsigned long long)__double_as_longlong(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long mm = 0;
    for (int w = 0; w < THREADS_PER_BLOCK / 32; ++w) mm = max(mm, mx[w]);
    atomicMax(&G.acc_max, mm);
  }
}

// After the loop: the peek step mu = x + peek alpha r (forcefield.py:1819-1820), the dipoles
// in FP64, the history push (forcefield.py:2005-2007) and mu + p for the energy pass.
template <typename T>
__global__ void k_cg_finish(Dev<T> a, double *mu, double *hist, int push) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  v4<T> x = a.X[i], r = a.R[i];
  T al = a.alpha[i];
  T pk = T(a.peek);
  if (a.peek != 0.0) { x.x += pk * r.x * al; x.y += pk * r.y * al; x.z += pk * r.z * al; }
  double m[3] = {double(x.x), double(x.y), double(x.z)};
  for (int c = 0; c < 3; ++c) mu[3 * i + c] = m[c];
  if (push) {
    size_t st = (size_t)a.nt * 3;
    for (int c = 0; c < 3; ++c) {
      size_t o = (size_t)3 * i + c;
      hist[3 * st + o] = hist[2 * st + o];
      hist[2 * st + o] = hist[st + o];
      hist[st + o] = hist[o];
      hist[o] = m[c];
    }
  }
}

__global__ void k_cg_state_out(const CGSys *cg, int nsys, int32_t *count, double *norm, int32_t *iters, double *resid,
                               unsigned *status, int push, double tol) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const CGSys &G = cg[s];
  if (push) { count[s] += 1; norm[s] = G.norm; }
  if (iters) iters[s] = G.it;
  if (resid) resid[s] = G.err;
  if (G.err > tol && !G.iel_ext) atomicOr(&status[s], 0x2u);  // an extended iEL step stops short of tol by design
}

// Per-system start of a solve: which predictor start applies (forcefield.py:1951-1966).
// mode 0: history predictor (compute); mode 1: the guess is the state's mu, plain start (energy,
// forcefield.py:2606-2612).
__global__ void k_cg_setup(CGSys *cg, int nsys, const int32_t *count, const double *norm, int K, int fused, int refresh,
                           int mode, cudaGraphConditionalHandle plain, int use_cond, int use_nn = 0) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  CGSys &G = cg[s];
  int c = count ? count[s] : 0;
  G.have = mode == 1 ? 1 : (K > 0 && c >= K);
  G.nn = use_nn && G.have;  // k_start1 adds the model's correction to the extrapolation
  G.fallback = 0;
  G.iel_ext = 0; G.iel_first = 0; G.maxit_s = -1; G.tol_s = -1.0;
  G.fused = mode == 0 && G.have && fused && (c % refresh) != 0;
  G.sweep2 = !G.fused;
  if (use_cond && G.sweep2) cudaGraphSetConditional(plain, 1u);  // the plain start's sweep runs (default 0)
  G.active = 0;
  G.norm = G.fused ? norm[s] : 1.0;
  G.acc_abs = 0; G.acc_rz = 0; G.acc_max = 0; G.acc_pap = 0; G.acc_num = 0;
}

// Energy-only start: x0 = the state's mu, first sweep at d = p.
template <typename T>
__global__ void k_energy_start(Dev<T> a, const double *mu) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  double4 p = a.pperm[i];
  v4<T> d, x;
  d.x = T(p.x); d.y = T(p.y); d.z = T(p.z); d.w = T(0);
  x.x = T(mu[3 * i]); x.y = T(mu[3 * i + 1]); x.z = T(mu[3 * i + 2]); x.w = T(0);
  a.D[i] = d;
  a.X[i] = x;
}

// ------------------------------------------------------------------ extended-Lagrangian dipoles
// iEL (forcefield.py:1452-1650, Niklasson's dissipative extended-Lagrangian Verlet): the
// auxiliary dipoles xl (K1, N, 3) FP64, newest first; warm-up steps (count < warmup) solve to tol,
// extended steps take x = xl[0]: 0-SCF mu = x + omega delta (no CG), SCF iel_iter CG iterations
// (to tol with 0) from x.

// Per system: first / warm-up / extended, the start the shared solver machinery takes (plain with
// its second sweep in the warm-up, fused from x otherwise), whether the first step starts from a
// given mu (any nonzero dipole of the system: one block per system), and the overrides of tol and
// max_iter (SCF with a set number of iterations: tol 0).
__global__ void k_iel_setup(CGSys *cg, const SysInfo *sys, int nsys, const int32_t *count, const double *norm, const double *mu,
                            int warmup, int scheme, int iel_iter, cudaGraphConditionalHandle plain, int use_cond) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int s = blockIdx.x;
  if (s >= nsys) return;
  const SysInfo &S = sys[s];
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  const int c = count[s];
  if (c == 0)
    for (int t = threadIdx.x; t < 3 * S.natom; t += blockDim.x)
      if (mu[3 * (size_t)S.atom0 + t] != 0.0) any = 1;
  __syncthreads();
  if (threadIdx.x) return;
  CGSys &G = cg[s];
  const int warm = c < warmup;
  G.iel_first = c == 0;
  G.iel_ext = !warm;
  G.have = c == 0 ? any : 1;
  G.nn = 0;
  G.fallback = 0;
  G.fused = !warm;
  G.sweep2 = warm;
  if (use_cond && warm) cudaGraphSetConditional(plain, 1u);  // the plain start's sweep runs (default 0)
  G.active = 0;
  G.norm = warm ? 1.0 : norm[s];
  G.tol_s = -1.0;
  G.maxit_s = -1;
  if (!warm && scheme == 2 && iel_iter > 0) { G.tol_s = 0.0; G.maxit_s = iel_iter; }
  G.acc_abs = 0; G.acc_rz = 0; G.acc_max = 0; G.acc_pap = 0; G.acc_num = 0;
}

// The start's first sweep: x0 = xl[0] (the first step: the given mu, or 0 and then alpha b), the
// dipoles p + x0 of the fused start or p of the plain one.
template <typename T>
__global__ void k_iel_start1(Dev<T> a, const double *xl, const double *mu) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  const CGSys &G = a.cg[a.sysid[i]];
  double x0[3] = {0, 0, 0};
  for (int c = 0; c < 3; ++c) x0[c] = G.iel_first ? (G.have ? mu[3 * (size_t)i + c] : 0.0) : xl[3 * (size_t)i + c];
  double4 p = a.pperm[i];
  v4<T> d, x;
  if (G.fused) { d.x = T(p.x + x0[0]); d.y = T(p.y + x0[1]); d.z = T(p.z + x0[2]); }
  else { d.x = T(p.x); d.y = T(p.y); d.z = T(p.z); }
  d.w = T(0);
  x.x = T(x0[0]); x.y = T(x0[1]); x.z = T(x0[2]); x.w = T(0);
  a.D[i] = d;
  a.X[i] = x;
}

// Solve M d = r for one molecule's block in FP64 (Gaussian elimination, partial pivoting), M =
// diag(1/alpha) + the same-molecule row tensors G1 I - G2 x x^T (forcefield.py:1530-1556).
template <typename T>
__device__ void iel_block_solve(const Dev<T> &a, int i0, int nb, double (*M)[25], double *d) {
  const int N = 3 * nb;
  for (int u = 0; u < N; ++u)
    for (int v = 0; v <= N; ++v) M[u][v] = 0.0;
  for (int li = 0; li < nb; ++li) {
    const int i = i0 + li;
    const v4<T> r = a.R[i];
    const double ia = 1.0 / double(a.alpha[i]);
    const double rr[3] = {double(r.x), double(r.y), double(r.z)};
    for (int c = 0; c < 3; ++c) { M[3 * li + c][3 * li + c] += ia; M[3 * li + c][N] = rr[c]; }
    const int nsp = a.rnsp[i];  // molecule partners first in every row
    const size_t base = (size_t)i * a.mc;
    for (int t = 0; t < nsp; ++t) {
      const int k = a.rk[base + t];
      const int lk = k - i0;
      if (lk < 0 || lk >= nb) continue;
      const double x[3] = {double(a.rx[base + t]), double(a.ry[base + t]), double(a.rz[base + t])};
      const double g1 = double(a.rg1[base + t]), g2 = double(a.rg2[base + t]);
      for (int u = 0; u < 3; ++u)
        for (int v = 0; v < 3; ++v) M[3 * li + u][3 * lk + v] += (u == v ? g1 : 0.0) - g2 * x[u] * x[v];
    }
  }
  for (int c = 0; c < N; ++c) {
    int pr = c;
    for (int u = c + 1; u < N; ++u)
      if (fabs(M[u][c]) > fabs(M[pr][c])) pr = u;
    if (pr != c)
      for (int v = 0; v <= N; ++v) { double t = M[c][v]; M[c][v] = M[pr][v]; M[pr][v] = t; }
    for (int u = c + 1; u < N; ++u) {
      const double f = M[u][c] / M[c][c];
      for (int v = c; v <= N; ++v) M[u][v] -= f * M[c][v];
    }
  }
  for (int c = N - 1; c >= 0; --c) {
    double acc = M[c][N];
    for (int v = c + 1; v < N; ++v) acc -= M[c][v] * d[v];
    d[c] = acc / M[c][c];
  }
}

// 0-SCF, one thread per molecule: for the extended systems delta = omega alpha r (Jacobi, and for
// molecules outside 2..8 atoms) or omega M^-1 r (block), mu = x + delta in FP64 (x = xl[0]), delta
// in Dl for the shadow energy, and max|delta| for the residual; zero delta elsewhere.
template <typename T>
__global__ void k_iel_delta(Dev<T> a, const double *xl, double omega, int block, double *mu, v4<T> *Dl) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmol) return;
  const int i0 = a.mol_start[m], nb = a.mol_start[m + 1] - i0;
  CGSys &G = a.cg[a.sysid[i0]];
  if (!G.iel_ext) {
    for (int i = i0; i < i0 + nb; ++i) Dl[i] = v4<T>{T(0), T(0), T(0), T(0)};
    return;
  }
  double d[24];
  double M[24][25];
  if (block && nb >= 2 && nb <= 8) {
    iel_block_solve(a, i0, nb, M, d);
  } else {
    for (int li = 0; li < nb && li < 8; ++li) {
      const v4<T> r = a.R[i0 + li];
      const double al = double(a.alpha[i0 + li]);
      d[3 * li] = al * double(r.x); d[3 * li + 1] = al * double(r.y); d[3 * li + 2] = al * double(r.z);
    }
  }
  double mx = 0.0;
  for (int li = 0; li < nb; ++li) {
    const int i = i0 + li;
    double dl[3];
    if (li < 8) {
      for (int c = 0; c < 3; ++c) dl[c] = omega * d[3 * li + c];
    } else {  // molecules above 8 atoms: Jacobi, atom by atom
      const v4<T> r = a.R[i];
      const double al = double(a.alpha[i]);
      dl[0] = omega * al * double(r.x); dl[1] = omega * al * double(r.y); dl[2] = omega * al * double(r.z);
    }
    for (int c = 0; c < 3; ++c) {
      mu[3 * (size_t)i + c] = xl[3 * (size_t)i + c] + dl[c];
      mx = fmax(mx, fabs(dl[c]));
    }
    Dl[i] = v4<T>{T(dl[0]), T(dl[1]), T(dl[2]), T(0)};
  }
  atomicMax(&G.acc_max, (unsigned long long)__double_as_longlong(mx));
}

// After the start (zscf: and the 0-SCF update): the extended 0-SCF systems' residual max|delta| /
// norm and no CG; *any over the systems that still iterate (warm-up solves, SCF from x), which
// with use_cond is also the captured loop's condition.
__global__ void k_iel_begin(CGSys *cg, int nsys, int *any, int zscf, cudaGraphConditionalHandle cond, int use_cond) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  __shared__ int act;
  if (threadIdx.x == 0) act = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < nsys; s += blockDim.x) {
    CGSys &G = cg[s];
    if (zscf && G.iel_ext) {
      G.err = __longlong_as_double((long long)G.acc_max) / G.norm;
      G.active = 0;
      G.acc_max = 0;
    }
    if (G.active) atomicOr(&act, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *any = act;
    if (use_cond) cudaGraphSetConditional(cond, act ? 1u : 0u);
  }
}

// After the solve: mu (the CG result with the peek step; 0-SCF extended systems: already written),
// the history push, and the auxiliary dipoles' step x_{n+1} = 2 Xh[0] - Xh[1] + kappa dx + a sum_k
// c_k Xh[k] with Xh = (mu, mu, ...) on the first step, xl with Xh[0] = mu in the warm-up, xl after,
// dx = mu - x on extended steps (0 in the warm-up); xl becomes (x_{n+1}, Xh[0], ..., Xh[K1 - 2]).
struct IelCoef {
  double kappa, a, c[10];
  int nc, K1, zscf;
};
template <typename T>
__global__ void k_iel_finish(Dev<T> a, double *mu, double *hist, double *xl, IelCoef co) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  const CGSys &G = a.cg[a.sysid[i]];
  const size_t st = (size_t)a.nt * 3;
  double m[3];
  if (G.iel_ext && co.zscf) {
    for (int c = 0; c < 3; ++c) m[c] = mu[3 * (size_t)i + c];
  } else {
    v4<T> x = a.X[i], r = a.R[i];
    const T al = a.alpha[i], pk = T(a.peek);
    if (a.peek != 0.0) { x.x += pk * r.x * al; x.y += pk * r.y * al; x.z += pk * r.z * al; }
    m[0] = double(x.x); m[1] = double(x.y); m[2] = double(x.z);
    for (int c = 0; c < 3; ++c) mu[3 * (size_t)i + c] = m[c];
  }
  for (int c = 0; c < 3; ++c) {
    const size_t o = (size_t)3 * i + c;
    hist[3 * st + o] = hist[2 * st + o];
    hist[2 * st + o] = hist[st + o];
    hist[st + o] = hist[o];
    hist[o] = m[c];
    double X[12];
    for (int j = 0; j < co.K1; ++j) X[j] = G.iel_first ? m[c] : ((j == 0 && !G.iel_ext) ? m[c] : xl[j * st + o]);
    double v = 2.0 * X[0] - X[1] + (G.iel_ext ? co.kappa * (m[c] - X[0]) : 0.0);
    if (co.a != 0.0)
      for (int k = 0; k < co.nc; ++k) v += co.a * co.c[k] * X[k];
    xl[o] = v;
    for (int j = 1; j < co.K1; ++j) xl[j * st + o] = X[j - 1];
  }
}

// ------------------------------------------------------------------ energy, forces, virial
// One group of LPA lanes per atom over its row: pair energies and their row gradients with the analytic
// kernels G0..G3 (forcefield.py:2294-2360), LJ rows, the row field at (q, d) (dE/dd), the pair
// virial sum g (x) x - gx (x) off; then the PME gradients of the atom: dU/dd and dU/dr through the
// spline derivatives (the autodiff of pme.py:390-411 written out).
// SHADOW (iEL/0-SCF, forcefield.py:2011-2045, 2294-2360): the energy is the shadow potential's,
// minus the pair and reciprocal energies of the dipoles Dl = delta alone (inside a molecule of 2..8
// atoms with the block preconditioner, the i-side delta scaled by a.iel_keep = 1 - 1/omega); their
// position gradients at fixed delta go to the forces, not to the virial (the fixed-mu strain
// derivative); the sums of |delta|^2 and |delta|^2 / (2 alpha) go to the energy accumulators.
template <typename T, int P, int MINB = 3, bool SHADOW = false, int LPA = 32>
__global__ void __launch_bounds__(8 * LPA, MINB * 32 / LPA) k_forces(Dev<T> a, const double *mu) {
  static_assert(LPA == 32 || LPA == 16 || LPA == 8, "lanes per atom");
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  __shared__ T sh[WARPS_PER_BLOCK][3][3][P];  // per atom of the block
  __shared__ double red[WARPS_PER_BLOCK][16];
  const int warp = threadIdx.x / LPA, lane = threadIdx.x % LPA;  // the atom's group of LPA lanes
  const unsigned gm = group_mask<LPA>();
  int s = a.wb_sys[blockIdx.x];
  int i = a.wb_atom0[blockIdx.x] + warp;
  const SysInfo &S = a.sys[s];
  bool valid = i < S.atom0 + S.natom;
  double vals[16];
  for (int k = 0; k < 16; ++k) vals[k] = 0.0;
  if (valid) {
    const BoxInfo &B = a.box[s];
    v4<T> di = a.D[i];
    T qi = a.q[i], rhi = a.rminh[i], sei = a.seps[i];
    int n = min(a.rn[i], a.mce), nsp = a.rnsp[i];
    size_t base = (size_t)i * a.mc;
    T gx0 = 0, gx1 = 0, gx2 = 0, gl0 = 0, gl1 = 0, gl2 = 0, fd0 = 0, fd1 = 0, fd2 = 0;
    T ee = 0, el = 0;
    T w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    T gs0 = 0, gs1 = 0, gs2 = 0;  // SHADOW: gradient of the delta-delta pair terms (forces only)
    v4<T> Dli = v4<T>{T(0), T(0), T(0), T(0)};
    bool blk_i = false;
    if constexpr (SHADOW) {
      Dli = a.Dl[i];
      const int msz = a.molend[i] - a.molfirst[i];
      blk_i = a.iel_keep_on && msz >= 2 && msz <= 8;
    }
    auto pair = [&](int k, T x, T y, T z, T G0, T G1, T G2, T G3, int t) {
      v4<T> dk = a.D[k];
      if constexpr (SHADOW) {
        const v4<T> Dk = a.Dl[k];
        const T wb = (blk_i && t < nsp) ? T(a.iel_keep) : T(1);  // molecule partners come first in a row
        const T Dix = wb * (Dli.x * x + Dli.y * y + Dli.z * z), Dkx = Dk.x * x + Dk.y * y + Dk.z * z;
        const T DiDk = wb * (Dli.x * Dk.x + Dli.y * Dk.y + Dli.z * Dk.z);
        ee += G2 * Dix * Dkx - G1 * DiDk;
        const T rad2 = -G3 * Dix * Dkx + G2 * DiDk;
        gs0 += rad2 * x + G2 * (wb * Dli.x * Dkx + Dk.x * Dix);
        gs1 += rad2 * y + G2 * (wb * Dli.y * Dkx + Dk.y * Dix);
        gs2 += rad2 * z + G2 * (wb * Dli.z * Dkx + Dk.z * Dix);
      }
      v4<T> pk = a.qls[k];  // q, R*/2, sqrt(eps) of the partner in one load
      T qk = pk.x;
      T dix = di.x * x + di.y * y + di.z * z;
      T dkx = dk.x * x + dk.y * y + dk.z * z;
      T didk = di.x * dk.x + di.y * dk.y + di.z * dk.z;
      const T qq = qi * qk, pp = dix * dkx;
      const T tt = qi * dkx - qk * dix;
      ee += qq * G0 + tt * G1 - G2 * pp + G1 * didk;
      const T radial = -qq * G1 - tt * G2 + G3 * pp - G2 * didk;
      // the gradient is radial x + u1 dk - u2 di, the field of (q_k, d_k) G1 dk - u2 x
      const T u1 = qi * G1 - G2 * dix, u2 = qk * G1 + G2 * dkx;
      T gxv = radial * x + u1 * dk.x - u2 * di.x;
      T gyv = radial * y + u1 * dk.y - u2 * di.y;
      T gzv = radial * z + u1 * dk.z - u2 * di.z;
      fd0 += G1 * dk.x - u2 * x; fd1 += G1 * dk.y - u2 * y; fd2 += G1 * dk.z - u2 * z;
      T kx = T(KE) * gxv, ky = T(KE) * gyv, kz = T(KE) * gzv;
      T ep = sei * pk.z;
      if (a.lj && t >= nsp && ep != T(0)) {  // LJ: not for molecule partners, nor pairs without an LJ term
        T rm = rhi + pk.y;
        T r2 = x * x + y * y + z * z;
        const T ir2 = T(1) / r2;
        T s2 = rm * rm * ir2, s6 = s2 * s2 * s2;
        el += ep * (s6 * s6 - T(2) * s6);
        T dl = ep * T(12) * (s6 - s6 * s6) * ir2;
        gl0 += dl * x; gl1 += dl * y; gl2 += dl * z;
        kx += dl * x; ky += dl * y; kz += dl * z;
      }
      gx0 += gxv; gx1 += gyv; gx2 += gzv;
      w[0] += kx * x; w[1] += kx * y; w[2] += kx * z;
      w[3] += ky * x; w[4] += ky * y; w[5] += ky * z;
      w[6] += kz * x; w[7] += kz * y; w[8] += kz * z;
    };
    if constexpr (sizeof(T) == 4) {
      // 16-byte loads of four consecutive entries of every row array
      const int4 *k4 = reinterpret_cast<const int4 *>(a.rk + base);
      const float4 *x4 = reinterpret_cast<const float4 *>(a.rx + base), *y4 = reinterpret_cast<const float4 *>(a.ry + base),
                   *z4 = reinterpret_cast<const float4 *>(a.rz + base), *h0 = reinterpret_cast<const float4 *>(a.rg0 + base),
                   *h1 = reinterpret_cast<const float4 *>(a.rg1 + base), *h2 = reinterpret_cast<const float4 *>(a.rg2 + base),
                   *h3 = reinterpret_cast<const float4 *>(a.rg3 + base);
      for (int t4 = lane; 4 * t4 < n; t4 += LPA) {
        int4 kk = __ldcs(k4 + t4);
        float4 xx = __ldcs(x4 + t4), yy = __ldcs(y4 + t4), zz = __ldcs(z4 + t4);
        float4 a0 = __ldcs(h0 + t4), a1 = __ldcs(h1 + t4), a2 = __ldcs(h2 + t4), a3 = __ldcs(h3 + t4);
        int t = 4 * t4;
        pair(kk.x, xx.x, yy.x, zz.x, a0.x, a1.x, a2.x, a3.x, t);
        if (t + 1 < n) pair(kk.y, xx.y, yy.y, zz.y, a0.y, a1.y, a2.y, a3.y, t + 1);
        if (t + 2 < n) pair(kk.z, xx.z, yy.z, zz.z, a0.z, a1.z, a2.z, a3.z, t + 2);
        if (t + 3 < n) pair(kk.w, xx.w, yy.w, zz.w, a0.w, a1.w, a2.w, a3.w, t + 3);
      }
    } else {
      for (int t = lane; t < n; t += LPA) {
        size_t o = base + t;
        pair(a.rk[o], a.rx[o], a.ry[o], a.rz[o], a.rg0[o], a.rg1[o], a.rg2[o], a.rg3[o], t);
      }
    }
    if (a.rnv) {  // split rows: the LJ pairs between elec_cutoff and cutoff
      const int nv = min(a.rnv[i], a.mc - a.mce);
      for (int t = lane; t < nv; t += LPA) {
        size_t o = base + a.mce + t;
        int k = a.rk[o];
        T x = a.rx[o], y = a.ry[o], z = a.rz[o];
        T rm = rhi + a.rminh[k], ep = sei * a.seps[k];
        T r2 = x * x + y * y + z * z;
        const T ir2 = T(1) / r2;
        T s2 = rm * rm * ir2, s6 = s2 * s2 * s2;
        el += ep * (s6 * s6 - T(2) * s6);
        T dl = ep * T(12) * (s6 - s6 * s6) * ir2;
        gl0 += dl * x; gl1 += dl * y; gl2 += dl * z;
        T kx = dl * x, ky = dl * y, kz = dl * z;
        w[0] += kx * x; w[1] += kx * y; w[2] += kx * z;
        w[3] += ky * x; w[4] += ky * y; w[5] += ky * z;
        w[6] += kz * x; w[7] += kz * y; w[8] += kz * z;
      }
    }
    // reciprocal gradients of the atom
    int4 b = a.base[i];
    v4<T> fr = a.frac[i];
    if (lane < 3) {
      T th[P], dth[P], d2[P];
      bspline<T, P, true>(lane == 0 ? fr.x : (lane == 1 ? fr.y : fr.z), th, dth, d2);
#pragma unroll
      for (int k = 0; k < P; ++k) { sh[warp][0][lane][k] = th[k]; sh[warp][1][lane][k] = dth[k]; sh[warp][2][lane][k] = d2[k]; }
    }
    __syncwarp(gm);
    T es[9];
#pragma unroll
    for (int bb = 0; bb < 3; ++bb)
#pragma unroll
      for (int aa = 0; aa < 3; ++aa) es[bb * 3 + aa] = T(B.Hinv[bb * 3 + aa] * S.K[aa]);
    T e0 = di.x * es[0] + di.y * es[3] + di.z * es[6];
    T e1 = di.x * es[1] + di.y * es[4] + di.z * es[7];
    T e2 = di.x * es[2] + di.y * es[5] + di.z * es[8];
    const T *phi = a.Phi + S.rgrid0;
    const int K1 = S.K[0], K2 = S.K[1], K3 = S.K[2];
    T ge0 = 0, ge1 = 0, ge2 = 0, gw0 = 0, gw1 = 0, gw2 = 0;
    if constexpr (SHADOW) {  // d/dr of the reciprocal energy of delta alone (its potential in Phi2)
      const T f0 = Dli.x * es[0] + Dli.y * es[3] + Dli.z * es[6];
      const T f1 = Dli.x * es[1] + Dli.y * es[4] + Dli.z * es[7];
      const T f2 = Dli.x * es[2] + Dli.y * es[5] + Dli.z * es[8];
      const T *phi2 = a.Phi2 + S.rgrid0;
      T h0 = 0, h1 = 0, h2 = 0;
      for (int p = lane; p < P * P * P; p += LPA) {
        int j1 = p / (P * P), j2 = (p / P) % P, j3 = p % P;
        int i1 = b.x + j1; if (i1 >= K1) i1 -= K1;
        int i2 = b.y + j2; if (i2 >= K2) i2 -= K2;
        int i3 = b.z + j3; if (i3 >= K3) i3 -= K3;
        T ph = phi2[((size_t)i1 * K2 + i2) * K3 + i3];
        T t1 = sh[warp][0][0][j1], t2 = sh[warp][0][1][j2], t3 = sh[warp][0][2][j3];
        T u1 = sh[warp][1][0][j1], u2 = sh[warp][1][1][j2], u3 = sh[warp][1][2][j3];
        T v1 = sh[warp][2][0][j1], v2 = sh[warp][2][1][j2], v3 = sh[warp][2][2][j3];
        h0 += ph * (f0 * v1 * t2 * t3 + f1 * u1 * u2 * t3 + f2 * u1 * t2 * u3);
        h1 += ph * (f0 * u1 * u2 * t3 + f1 * t1 * v2 * t3 + f2 * t1 * u2 * u3);
        h2 += ph * (f0 * u1 * t2 * u3 + f1 * t1 * u2 * u3 + f2 * t1 * t2 * v3);
      }
      // the pair part is KE (gx + gs); the reciprocal part of -U_rec(0, delta) enters with a minus sign
      gs0 = gs0 - h0 * es[0] - h1 * es[1] - h2 * es[2];
      gs1 = gs1 - h0 * es[3] - h1 * es[4] - h2 * es[5];
      gs2 = gs2 - h0 * es[6] - h1 * es[7] - h2 * es[8];
    }
    for (int p = lane; p < P * P * P; p += LPA) {
      int j1 = p / (P * P), j2 = (p / P) % P, j3 = p % P;
      int i1 = b.x + j1; if (i1 >= K1) i1 -= K1;
      int i2 = b.y + j2; if (i2 >= K2) i2 -= K2;
      int i3 = b.z + j3; if (i3 >= K3) i3 -= K3;
      T ph = phi[((size_t)i1 * K2 + i2) * K3 + i3];
      T t1 = sh[warp][0][0][j1], t2 = sh[warp][0][1][j2], t3 = sh[warp][0][2][j3];
      T u1 = sh[warp][1][0][j1], u2 = sh[warp][1][1][j2], u3 = sh[warp][1][2][j3];
      T v1 = sh[warp][2][0][j1], v2 = sh[warp][2][1][j2], v3 = sh[warp][2][2][j3];
      ge0 += ph * u1 * t2 * t3;
      ge1 += ph * t1 * u2 * t3;
      ge2 += ph * t1 * t2 * u3;
      gw0 += ph * (qi * u1 * t2 * t3 + e0 * v1 * t2 * t3 + e1 * u1 * u2 * t3 + e2 * u1 * t2 * u3);
      gw1 += ph * (qi * t1 * u2 * t3 + e0 * u1 * u2 * t3 + e1 * t1 * v2 * t3 + e2 * t1 * u2 * u3);
      gw2 += ph * (qi * t1 * t2 * u3 + e0 * u1 * t2 * u3 + e1 * t1 * u2 * u3 + e2 * t1 * t2 * v3);
    }
    T red_in[24] = {gx0, gx1, gx2, gl0, gl1, gl2, fd0, fd1, fd2, ee, el, ge0, ge1, ge2, gw0, gw1, gw2,
                    w[0], w[1], w[2], w[3], w[4], w[5], w[6]};
#pragma unroll
    for (int k = 0; k < 24; ++k) red_in[k] = group_sum<T, LPA>(red_in[k], gm);
    T w7 = group_sum<T, LPA>(w[7], gm), w8 = group_sum<T, LPA>(w[8], gm);
    if constexpr (SHADOW) { gs0 = group_sum<T, LPA>(gs0, gm); gs1 = group_sum<T, LPA>(gs1, gm); gs2 = group_sum<T, LPA>(gs2, gm); }
    if (lane == 0) {
      double gd[3], gr[3];
      for (int bb = 0; bb < 3; ++bb) {
        gd[bb] = double(red_in[11]) * double(es[bb * 3 + 0]) + double(red_in[12]) * double(es[bb * 3 + 1]) + double(red_in[13]) * double(es[bb * 3 + 2]);
        gr[bb] = double(red_in[14]) * double(es[bb * 3 + 0]) + double(red_in[15]) * double(es[bb * 3 + 1]) + double(red_in[16]) * double(es[bb * 3 + 2]);
      }
      double d3[3] = {double(di.x), double(di.y), double(di.z)};
      double gx[3] = {double(red_in[0]), double(red_in[1]), double(red_in[2])};
      double gl[3] = {double(red_in[3]), double(red_in[4]), double(red_in[5])};
      double fd[3] = {double(red_in[6]), double(red_in[7]), double(red_in[8])};
      double4 of = a.off[i];
      double ofs[3] = {of.x, of.y, of.z};
      double cs = a.c_self;
      double dE[3];
      const double gsh[3] = {double(gs0), double(gs1), double(gs2)};
      for (int c = 0; c < 3; ++c) {
        a.forces[3 * i + c] = -(KE * gx[c] + gl[c] + KE * gr[c] + (SHADOW ? KE * gsh[c] : 0.0));
        dE[c] = KE * (fd[c] + gd[c] - cs * d3[c]);
      }
      if constexpr (SHADOW) {
        const double dl2 = double(Dli.x) * double(Dli.x) + double(Dli.y) * double(Dli.y) + double(Dli.z) * double(Dli.z);
        vals[13] = dl2;
        vals[14] = dl2 / (2.0 * double(a.alpha[i]));
      }
      a.dEdd[i] = make_double4(dE[0], dE[1], dE[2], 0);
      vals[0] = double(red_in[9]);
      vals[1] = double(red_in[10]);
      vals[2] = d3[0] * d3[0] + d3[1] * d3[1] + d3[2] * d3[2];
      if (a.induce && mu) {
        double m0 = mu[3 * i], m1 = mu[3 * i + 1], m2 = mu[3 * i + 2];
        vals[3] = (m0 * m0 + m1 * m1 + m2 * m2) / (2.0 * double(a.alpha[i]));
      }
      // virial: 1/2 sum_rows g (x) x - (KE gx + gl) (x) off - KE (dU/dr (x) off + dU/dd (x) d)
      double wsum[9] = {double(red_in[17]), double(red_in[18]), double(red_in[19]), double(red_in[20]), double(red_in[21]),
                        double(red_in[22]), double(red_in[23]), double(w7), double(w8)};
      for (int aa = 0; aa < 3; ++aa)
        for (int bb = 0; bb < 3; ++bb)
          vals[4 + aa * 3 + bb] = 0.5 * wsum[aa * 3 + bb] - (KE * gx[aa] + gl[aa]) * ofs[bb] - KE * (gr[aa] * ofs[bb] + gd[aa] * d3[bb]);
    }
  }
  constexpr int NV = SHADOW ? 15 : 13;
  if (lane == 0)
    for (int k = 0; k < NV; ++k) red[warp][k] = vals[k];
  __syncthreads();
  if (threadIdx.x < NV) {
    double v = 0;
    for (int w2 = 0; w2 < WARPS_PER_BLOCK; ++w2) v += red[w2][threadIdx.x];
    EnergyAcc &E = a.eacc[s];
    double *dst = threadIdx.x == 0 ? &E.e_pair : threadIdx.x == 1 ? &E.e_lj : threadIdx.x == 2 ? &E.d2
                  : threadIdx.x == 3 ? &E.upol : threadIdx.x == 13 ? &E.dd2 : threadIdx.x == 14 ? &E.dda
                  : &E.vir[threadIdx.x - 4];
    atomicAdd(dst, v);
  }
}

// Covalent-dipole frames: p_i = sum c unit(r_j - r_i); the pull-back of dE/dd_i onto r_i and r_j
// (the vector-Jacobian product of forcefield.py:2412).  One thread per covalent dipole.
template <typename T>
__global__ void k_cov_forces(Dev<T> a) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.ncov || !a.perm) return;
  int i = a.cov_i_flat[m], j = a.cov_j_flat[m];
  const BoxInfo &B = a.box[a.sysid[i]];
  double vx = a.pos[3 * j] - a.pos[3 * i], vy = a.pos[3 * j + 1] - a.pos[3 * i + 1], vz = a.pos[3 * j + 2] - a.pos[3 * i + 2];
  min_image(vx, vy, vz, B.H);
  double l = sqrt(vx * vx + vy * vy + vz * vz);
  double ux = vx / l, uy = vy / l, uz = vz / l;
  double4 g = a.dEdd[i];
  double ug = ux * g.x + uy * g.y + uz * g.z;
  double c = a.cov_c_flat[m] / l;
  double gx = c * (g.x - ux * ug), gy = c * (g.y - uy * ug), gz = c * (g.z - uz * ug);
  atomicAdd(&a.forces[3 * j], -gx); atomicAdd(&a.forces[3 * j + 1], -gy); atomicAdd(&a.forces[3 * j + 2], -gz);
  atomicAdd(&a.forces[3 * i], gx); atomicAdd(&a.forces[3 * i + 1], gy); atomicAdd(&a.forces[3 * i + 2], gz);
}

// Energies and virial of every system (forcefield.py:2011-2045, 2420-2430, lj.py:87-114):
// E_elec = KE [rows/2 + U_rec + U_self + U_bg + U_pol], E_vdw = rows/2 + tail.
__global__ void k_energy_finish(const SysInfo *sys, const BoxInfo *box, const EnergyAcc *E, int nsys, double beta, double c_self,
                                double cutoff, int lj, int lj_lrc, int induce, double *energy, double *virial, unsigned *status,
                                const EnergyAcc *E2 = nullptr, double omega = 1.0) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  const EnergyAcc &e = E[s];
  const SysInfo &S = sys[s];
  double vol = box[s].vol;
  double uself = -(beta / SQRT_PI) * S.sum_q2 - 0.5 * c_self * e.d2;
  double urec_delta = 0.0;
  if (E2) {  // iEL/0-SCF shadow energy (forcefield.py:2037-2042)
    uself += 0.5 * c_self * e.dd2 - (1.0 - 1.0 / omega) * e.dda;
    urec_delta = E2[s].vinf[0];
  }
  double ubg = -PI * S.sum_q * S.sum_q / (2.0 * vol * beta * beta);
  double upol = induce ? e.upol : 0.0;
  double elec = 0.5 * KE * e.e_pair + KE * (e.vinf[0] - urec_delta + uself + ubg + upol);
  double tail = (lj && lj_lrc) ? -2.0 * PI * S.tail_sb / (3.0 * vol * cutoff * cutoff * cutoff) : 0.0;
  double vdw = 0.5 * e.e_lj + tail;
  if (energy) {
    energy[3 * s] = elec;
    energy[3 * s + 1] = vdw;
    energy[3 * s + 2] = elec + vdw;
  }
  if (!isfinite(elec + vdw)) atomicOr(&status[s], 0x4u);
  if (virial) {
    double W[9];
    for (int k = 0; k < 9; ++k) W[k] = e.vir[k];
    W[0] += KE * e.vinf[1]; W[4] += KE * e.vinf[2]; W[8] += KE * e.vinf[3];
    W[1] += KE * e.vinf[4]; W[3] += KE * e.vinf[4];
    W[2] += KE * e.vinf[5]; W[6] += KE * e.vinf[5];
    W[5] += KE * e.vinf[6]; W[7] += KE * e.vinf[6];
    for (int c = 0; c < 3; ++c) W[4 * c] += -KE * ubg - 2.0 * tail;
    for (int k = 0; k < 9; ++k) virial[9 * s + k] = W[k];
  }
}

// d = p + mu (energy pass), in T.
template <typename T>
__global__ void k_total_dipoles(Dev<T> a, const double *mu) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  // the energy accumulators of the pass start at zero
  constexpr int NACC = sizeof(EnergyAcc) / sizeof(double);
  for (int t = i; t < NACC * a.nsys; t += gridDim.x * blockDim.x) reinterpret_cast<double *>(a.eacc)[t] = 0.0;
  if (i >= a.nt) return;
  double4 p = a.pperm[i];
  double m0 = mu ? mu[3 * i] : 0.0, m1 = mu ? mu[3 * i + 1] : 0.0, m2 = mu ? mu[3 * i + 2] : 0.0;
  v4<T> d;
  d.x = T(p.x + m0); d.y = T(p.y + m1); d.z = T(p.z + m2); d.w = T(0);
  a.D[i] = d;
}

// Copy of a (N, 3) FP64 array into v4<T> (pgm_field input).
template <typename T>
__global__ void k_load_vec(Dev<T> a, const double *v, v4<T> *out) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  v4<T> d;
  d.x = T(v[3 * i]); d.y = T(v[3 * i + 1]); d.z = T(v[3 * i + 2]); d.w = T(0);
  out[i] = d;
}

template <typename T>
__global__ void k_store_vec(Dev<T> a, const v4<T> *in, double *v) {
  pdl_enter();  // launched as a programmatic dependent of the previous kernel
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.nt) return;
  v4<T> d = in[i];
  v[3 * i] = double(d.x); v[3 * i + 1] = double(d.y); v[3 * i + 2] = double(d.z);
}

}  // namespace pgm
