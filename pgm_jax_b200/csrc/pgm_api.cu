// pgm_api.cu -- host side of the B200 pGM engine: the handle, the buffers, the launch sequence
// of a step and the C ABI declared in include/pgm_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/pgm_b200.h"
#include "pgm_kernels.cuh"

namespace pgmmp_engine {  // the message-passing model of the learned guess (pgm_mpnn.cu)
size_t work_bytes(int n);
cudaError_t set_weights(const float *flat, void *work, int n, cudaStream_t st);
cudaError_t predict(const float *flat, void *work, const float *inv, const float *vec, const float4 *edges, const int *ecount,
                    int emax, int n, float sigma, float rg, float *mu, cudaStream_t st, int prio);
}  // namespace pgmmp_engine

namespace {

thread_local std::string g_err;

struct CudaError {
  std::string msg;
};

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) throw CudaError{std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

template <typename X>
struct DBuf {
  X *p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free();
    n = count;
    if (count) CK(cudaMalloc(&p, sizeof(X) * count));
  }
  void upload(const std::vector<X> &v) {
    alloc(v.size());
    if (!v.empty()) CK(cudaMemcpy(p, v.data(), sizeof(X) * v.size(), cudaMemcpyHostToDevice));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { free(); }
};

// Host copy of the B-spline recursion at f = 0 and the moduli (pme.py:106-131).
void host_bspline0(int order, double *th) {
  std::vector<double> d(order + 1, 0.0);
  double f = 0.0;
  d[0] = 1.0 - f;
  d[1] = f;
  for (int n = 3; n <= order; ++n) {
    double div = 1.0 / (n - 1.0);
    d[n - 1] = div * f * d[n - 2];
    for (int k = 1; k < n - 1; ++k) d[n - k - 1] = div * ((f + k) * d[n - k - 2] + (n - k - f) * d[n - k - 1]);
    d[0] = div * (1.0 - f) * d[0];
  }
  for (int k = 0; k < order; ++k) th[k] = d[k];
}

std::vector<double> host_moduli(int K, int order) {
  std::vector<double> th(order), mod(K);
  host_bspline0(order, th.data());
  for (int m = 0; m < K; ++m) {
    double c = 0, s = 0;
    for (int j = 0; j < order; ++j) {
      double arg = 2.0 * M_PI * m * j / K;
      c += th[j] * std::cos(arg);
      s += th[j] * std::sin(arg);
    }
    mod[m] = c * c + s * s;
  }
  for (int m = 0; m < K; ++m)
    if (mod[m] < 1e-7) mod[m] = 0.5 * (mod[(m - 1 + K) % K] + mod[(m + 1) % K]);
  return mod;
}

// Radices of a length-K FFT (4s first, then 2, 3, 5); empty if K has another factor.
std::vector<int> radices(int K) {
  std::vector<int> r;
  while (K % 4 == 0) { r.push_back(4); K /= 4; }
  while (K % 2 == 0) { r.push_back(2); K /= 2; }
  while (K % 3 == 0) { r.push_back(3); K /= 3; }
  while (K % 5 == 0) { r.push_back(5); K /= 5; }
  if (K != 1) r.clear();
  return r;
}

struct EngineBase {
  virtual ~EngineBase() {
    if (host_scratch) cudaFree(host_scratch);
  }
  virtual void compute(cudaStream_t st, const double *pos, const double *box, const int32_t *idx, int idx_width,
                       PgmInduction *ind, PgmOutputs *out) = 0;
  virtual void energy(cudaStream_t st, const double *pos, const double *box, const int32_t *idx, int idx_width,
                      PgmInduction *ind, double *energy, int32_t *iters, uint32_t *status) = 0;
  virtual void field(cudaStream_t st, const double *pos, const double *box, int with_q, const double *d, double *out) = 0;
  virtual void fixed_mu(cudaStream_t st, const double *pos, const double *box, const int32_t *idx, int idx_width,
                        const double *mu, double *energy, double *forces, double *virial, uint32_t *status) = 0;
  virtual void set_capacity(int mc) = 0;
  virtual bool set_elec_capacity(int c) = 0;
  virtual int elec_capacity() const = 0;
  virtual int max_vdw_count() = 0;
  virtual void set_nn(const float *w, float sigma, float rg) = 0;
  virtual void set_mpnn(const float *w, int nparam, float sigma, float rg) = 0;
  virtual void nn_graph(cudaStream_t st, float4 *edges, int *counts, int emax) = 0;
  virtual void set_nn_fallback(double factor) = 0;
  virtual void set_tuning(int rowfield_lanes, int forces_blocks, int sweep_early, int rowfield_grid) = 0;
  virtual void autotune(cudaStream_t st) = 0;
  virtual PgmTuning tuning() const = 0;
  virtual void nn_fallback_stats(long long *fallbacks, double *ref_err) = 0;
  virtual void nn_features(cudaStream_t st, const double *pos, const double *box, const double *hist, const float *bl_prev,
                           float *bl_out, float *inv, float *vec) = 0;
  virtual void set_list_capacity(int c) = 0;
  virtual int list_capacity() const = 0;
  virtual long long list_rebuilds() = 0;
  virtual int capacity() const = 0;
  virtual int max_count() = 0;
  virtual long long launches_per_iteration() const = 0;
  virtual double profile(cudaStream_t st, int which, int reps) = 0;
  virtual bool has_hist() const = 0;
  virtual long long row_pairs() = 0;
  int nt = 0, nsys = 0;
  int iel_len = 0;  // auxiliary dipoles kept by an iEL state (0: no iEL)
  double *host_scratch = nullptr;  // device block of pgm_compute_host (allocated on first use)
  size_t host_scratch_bytes = 0;
  long long launches = 0;
  int unrolled = 0;  // CG iterations unrolled in front of the while node of the last capture
  long long generation = 0;  // bumped when device buffers are reallocated (captured graphs go stale)
};

// Mesh lengths with a compiled FFT plan (others run the runtime-length kernels).
template <typename F>
void with_fft_len(int L, F &&f) {
  switch (L) {
    case 32: f(std::integral_constant<int, 32>{}); break;
    case 48: f(std::integral_constant<int, 48>{}); break;
    case 64: f(std::integral_constant<int, 64>{}); break;
    case 72: f(std::integral_constant<int, 72>{}); break;
    case 96: f(std::integral_constant<int, 96>{}); break;
    case 128: f(std::integral_constant<int, 128>{}); break;
    case 192: f(std::integral_constant<int, 192>{}); break;
    default: f(std::integral_constant<int, 0>{}); break;
  }
}

// The systems of one FFT pass launch: same mesh length along the pass's axis.
struct FftGroup {
  int K = 0, ng = 0, ntiles = 0;
  size_t smem = 0;
  DBuf<int> sys, tile0;
};

// Autotuner choices, shared by the handles of one process with the same precision, spline
// order, atoms, row capacity and grid size (timed once per such shape).
struct TuneKey {
  int tsize, order, nt, mc;
  long long rgrid;
  bool operator<(const TuneKey &o) const {
    return std::tie(tsize, order, nt, mc, rgrid) < std::tie(o.tsize, o.order, o.nt, o.mc, o.rgrid);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, PgmTuning> g_tune_cache;

template <typename T, int P>
struct Engine : EngineBase {
  PgmSettings set;
  std::vector<pgm::SysInfo> hsys;
  int nmol_total = 0, ncell = 0, ncov = 0, mc = 0, mc_auto = 0, cc = 0, cc_auto = 0;
  // split rows (elec_cutoff < cutoff): electrostatic part [0, mce) of every row, LJ part [mce, mc)
  double rc_e = 0.0;
  bool split = false;
  int mce = 0, mce_auto = 0;
  DBuf<int> rnv;
  double skin = 0.0;
  long long rgrid = 0, cgrid = 0;
  std::vector<std::unique_ptr<FftGroup>> gx, gy, gz, gp;  // k3, k2, k1 passes; plane passes (k3 + k2)
  int nwblk = 0, ntblk = 0;
  std::vector<int> natoms;

  DBuf<pgm::SysInfo> d_sys;
  DBuf<pgm::BoxInfo> d_box;
  DBuf<pgm::CGSys> d_cg;
  DBuf<pgm::EnergyAcc> d_eacc;
  DBuf<unsigned> d_status;
  DBuf<int> wb_sys, wb_atom0, tb_sys, tb_atom0;
  DBuf<int> sysid, molid, molfirst, molend, mol_start, cov_start, cov_j, cov_i_flat, cov_j_flat;
  DBuf<T> q, radius, alpha, ialpha, rminh, seps;
  DBuf<pgm::v4<T>> qls;
  DBuf<double> mass, cov_c, cov_c_flat, bmod;
  DBuf<int4> base;
  DBuf<pgm::v4<T>> frac, X, R, Z, Pv, AP, Bv, D, Fv, Fpv;
  DBuf<double4> pperm, off, dEdd;
  DBuf<int> cell_of, slot_of, cell_count, cell_start, cell_atoms;
  DBuf<double4> spos, pos_ref, pos4;
  DBuf<float4> pos4f;  // mixed precision: wrapped FP32 positions for the row build
  DBuf<int> cand, ncand, nb_flag;
  DBuf<long long> nb_builds;
  DBuf<int> rn, rnsp, rk, dmax, dany;
  DBuf<unsigned> cg_done;  // blocks of the fused CG update that have finished (the last one checks)
  DBuf<T> rx, ry, rz, rg0, rg1, rg2, rg3;
  DBuf<T> Q, Phi, Ginf;
  DBuf<pgm::c2<T>> C, tw;
  DBuf<double> mu_tmp, forces_tmp, energy_tmp;
  DBuf<float> nn_w, nn_inv, nn_vec, nn_mu, nn_chan;  // learned guess: model and per-atom features
  DBuf<__nv_bfloat16> nn_wb;  // the model's weight matrices in BF16 (converted when the model is set)
  bool mp_on = false;         // the message-passing model instead of the per-atom MLP
  DBuf<float> mp_w;           // its FP32 parameters
  DBuf<unsigned char> mp_work;  // its activations and BF16 weights
  bool nn_on = false;
  // extended-Lagrangian dipoles: the recurrence's coefficients, delta, the reciprocal potential of
  // delta alone and its energy accumulators (shadow potential)
  pgm::IelCoef iel_co{};
  int iel_warmup = 0;
  bool iel_shadow = false;
  DBuf<pgm::v4<T>> Dl;
  DBuf<T> Phi2;
  DBuf<pgm::EnergyAcc> d_eacc2;
  PgmTuning tune{32, 3};     // kernel variants in use (autotuned at the first direct step unless fixed)
  bool tune_fixed = false;
  double nn_fb_factor = 2.0;  // learned guess: fall back to x4 when its start residual is above this x the record
  DBuf<int> dfb;              // some system falls back (the host-driven solve reads it)
  int last_iters = 0;  // CG iterations of the last host-driven solve (sizes the unrolled part of a capture)
  const double *last_hist = nullptr;  // the history of the last predictor solve (profiling)
  DBuf<float4> nn_bl;  // the graph's permanent field of the last solve (for the change channel)
  DBuf<int> nn_valid;  // nn_bl holds a previous step
  DBuf<float4> nn_e4;  // the learned guess's graph edges per atom (written by the row build)
  DBuf<float2> nn_g;  // G1, G2 of each edge
  DBuf<int> nn_ne;
  // local preconditioner (set.local_niter > 0): the short entries (entry-major) and their counts,
  // the inner CG's vectors
  static constexpr int SH_MAX = 48;
  DBuf<int> sh_n, c_k;
  DBuf<T> c_x, c_y, c_z, c_g1, c_g2;
  DBuf<pgm::v4<T>> LRR, LZZ, LP0, LP1, DRv;
  static constexpr int NN_EMAX = 128;
  // lanes per atom of the spread, the PME gather, the force pass, the row build and the learned
  // guess's channel pass (32: a warp per atom; 16, 8: two, four atoms per warp)
  static constexpr int SPREAD_LPA = 8, GATHER_LPA = 8, FORCES_LPA = 8, ROWS_LPA = 32, CHAN_LPA = 32;
  // the row build evaluates the kernels after its scan (true) or in it, on the keeping lanes (false)
  static constexpr bool ROWS_TWO_PHASE = true;
  float nn_sigma = 2e-4f, nn_rg = 0.5f;  // until pgm_set_nn_model
  int *h_any = nullptr;
  const double *last_pos = nullptr;
  cudaStream_t side = nullptr, aux = nullptr, aux_b = nullptr, nn_st = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_fork_b = nullptr, ev_join_b = nullptr, ev_nn_fork = nullptr,
              ev_nn_join = nullptr;
  bool nn_forked = false;  // the learned guess of this step runs on nn_st (joined before the solve's start)
  bool in_body = false;  // enqueueing the body of a conditional node (its own capture sequence)
  bool overlap = true;  // row field on a second stream beside the FFT chain
  int prio_hi = 0;      // the device's highest stream priority (the learned guess's kernels)
  int nsm = 148;        // multiprocessors of the device
  long long per_iter = 0;

  ~Engine() {
    if (h_any) cudaFreeHost(h_any);
    if (side) cudaStreamDestroy(side);
    if (aux) cudaStreamDestroy(aux);
    if (aux_b) cudaStreamDestroy(aux_b);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_fork_b) cudaEventDestroy(ev_fork_b);
    if (ev_join_b) cudaEventDestroy(ev_join_b);
    if (nn_st) cudaStreamDestroy(nn_st);
    if (ev_nn_fork) cudaEventDestroy(ev_nn_fork);
    if (ev_nn_join) cudaEventDestroy(ev_nn_join);
  }

  pgm::Dev<T> dev(const double *pos, const int32_t *idx, int idx_width, double *forces, unsigned *status) {
    pgm::Dev<T> a;
    std::memset(&a, 0, sizeof(a));
    a.nsys = nsys; a.nt = nt; a.nmol = nmol_total; a.mc = mc; a.ncell = ncell; a.ncov = ncov;
    a.order = P;
    a.induce = (set.elec == 2 || set.elec == 3);
    a.perm = (set.elec == 1 || set.elec == 3);
    a.lj = set.vdw == 1;
    a.lj_lrc = set.lj_lrc;
    a.beta = set.ewald_beta; a.cutoff = set.cutoff;
    a.c_self = 4.0 * std::pow(set.ewald_beta, 3) / (3.0 * pgm::SQRT_PI);
    a.tol = set.dipole_tol; a.peek = set.peek; a.max_iter = set.max_iter;
    a.sys = d_sys.p; a.box = d_box.p; a.cg = d_cg.p; a.eacc = d_eacc.p; a.status = status;
    a.wb_sys = wb_sys.p; a.wb_atom0 = wb_atom0.p; a.tb_sys = tb_sys.p; a.tb_atom0 = tb_atom0.p;
    a.sysid = sysid.p; a.molid = molid.p; a.molfirst = molfirst.p; a.molend = molend.p; a.mol_start = mol_start.p;
    a.q = q.p; a.radius = radius.p; a.alpha = alpha.p; a.ialpha = ialpha.p; a.rminh = rminh.p; a.seps = seps.p;
    a.qls = qls.p;
    a.mass = mass.p;
    a.cov_start = cov_start.p; a.cov_j = cov_j.p; a.cov_i_flat = cov_i_flat.p; a.cov_j_flat = cov_j_flat.p;
    a.cov_c = cov_c.p; a.cov_c_flat = cov_c_flat.p;
    a.pos = pos;
    a.base = base.p; a.frac = frac.p; a.pperm = pperm.p; a.off = off.p;
    a.cell_of = cell_of.p; a.slot_of = slot_of.p; a.cell_count = cell_count.p; a.cell_start = cell_start.p;
    a.cell_atoms = cell_atoms.p;
    a.spos = spos.p;
    a.skin = skin; a.cc = cc; a.nb_flag = nb_flag.p; a.nb_builds = nb_builds.p; a.cand = cand.p; a.ncand = ncand.p;
    a.pos_ref = pos_ref.p; a.pos4 = pos4.p; a.pos4f = pos4f.p;
    a.idx = idx; a.idx_width = idx_width;
    a.rn = rn.p; a.rnsp = rnsp.p; a.rk = rk.p;
    a.rx = rx.p; a.ry = ry.p; a.rz = rz.p; a.rg0 = rg0.p; a.rg1 = rg1.p; a.rg2 = rg2.p; a.rg3 = rg3.p;
    a.max_count = dmax.p;
    a.mce = mce; a.rnv = split ? rnv.p : nullptr; a.rce2 = rc_e * rc_e;
    a.nn_e4 = nn_e4.p; a.nn_g = nn_g.p; a.nn_ne = nn_ne.p; a.nn_emax = NN_EMAX; a.nn_rg2 = nn_rg * nn_rg;
    if (set.local_niter > 0) {
      a.sh_n = sh_n.p; a.sh_max = SH_MAX; a.lc2 = set.local_cut * set.local_cut;
      a.c_k = c_k.p; a.c_x = c_x.p; a.c_y = c_y.p; a.c_z = c_z.p; a.c_g1 = c_g1.p; a.c_g2 = c_g2.p;
      a.LRR = LRR.p; a.LZZ = LZZ.p; a.LP0 = LP0.p; a.LP1 = LP1.p; a.DR = DRv.p;
    }
    a.X = X.p; a.R = R.p; a.Z = Z.p; a.P = Pv.p; a.AP = AP.p; a.B = Bv.p; a.D = D.p; a.F = Fv.p; a.Fp = Fpv.p;
    a.Q = Q.p; a.Phi = Phi.p; a.Ginf = Ginf.p; a.C = C.p; a.tw = tw.p; a.bmod = bmod.p;
    a.forces = forces; a.dEdd = dEdd.p;
    a.Dl = Dl.p; a.Phi2 = Phi2.p;
    const double om = set.iel_omega > 0 ? set.iel_omega : 1.0;
    a.iel_keep = 1.0 - 1.0 / om;
    a.iel_keep_on = set.iel == 1 && set.iel_precond == 0;
    return a;
  }

  void init(const PgmSettings *s, const PgmSystemDesc *systems, int n) {
    set = *s;
    nsys = n;
    hsys.resize(n);
    std::vector<int> h_sysid, h_molid, h_molfirst, h_molend, h_molstart, h_covstart, h_covj, h_covi_flat, h_covj_flat;
    std::vector<T> h_q, h_rad, h_al, h_ial, h_rh, h_se;
    std::vector<double> h_mass, h_covc, h_covc_flat, h_bmod;
    std::vector<pgm::c2<T>> h_tw;
    std::vector<int> twK;
    std::vector<int> tw_off;
    int atom0 = 0, mol0 = 0, cell0 = 0;
    double rho_max = 0;
    long long rg = 0, cg = 0;
    auto tw_for = [&](int K) {
      for (size_t t = 0; t < twK.size(); ++t)
        if (twK[t] == K) return tw_off[t];
      int o = (int)h_tw.size();
      for (int m = 0; m < K; ++m) {
        pgm::c2<T> c;
        c.x = T(std::cos(2.0 * M_PI * m / K));
        c.y = T(-std::sin(2.0 * M_PI * m / K));
        h_tw.push_back(c);
      }
      twK.push_back(K);
      tw_off.push_back(o);
      return o;
    };
    for (int si = 0; si < n; ++si) {
      const PgmSystemDesc &d = systems[si];
      pgm::SysInfo &S = hsys[si];
      std::memset(&S, 0, sizeof(S));
      S.atom0 = atom0; S.natom = d.n_atoms; S.mol0 = mol0; S.nmol = d.n_mol;
      for (int a = 0; a < 3; ++a) S.K[a] = d.pme_grid[a];
      S.K3h = S.K[2] / 2 + 1;
      rg = (rg + 63) / 64 * 64;  // every system's grids start 256-byte aligned (16-byte vector atomics)
      cg = (cg + 63) / 64 * 64;
      S.rgrid0 = rg; S.cgrid0 = cg;
      rg += (long long)S.K[0] * S.K[1] * S.K[2];
      cg += (long long)S.K[0] * S.K[1] * S.K3h;
      for (int a = 0; a < 3; ++a) {
        std::vector<int> r = radices(S.K[a]);
        S.nst[a] = (int)r.size();
        for (size_t k = 0; k < r.size(); ++k) S.rad[a][k] = r[k];
        S.tw[a] = tw_for(S.K[a]);
        S.mod0[a] = (int)h_bmod.size();
        std::vector<double> mm = host_moduli(S.K[a], P);
        h_bmod.insert(h_bmod.end(), mm.begin(), mm.end());
      }
      // cell grid from the plane heights of box0: cells at least rc / 2 thick
      const double *H = d.box0;
      double det = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) + H[2] * (H[3] * H[7] - H[4] * H[6]);
      double vol = std::fabs(det);
      auto cross = [&](int i, int j, double *o) {
        o[0] = H[i * 3 + 1] * H[j * 3 + 2] - H[i * 3 + 2] * H[j * 3 + 1];
        o[1] = H[i * 3 + 2] * H[j * 3 + 0] - H[i * 3 + 0] * H[j * 3 + 2];
        o[2] = H[i * 3 + 0] * H[j * 3 + 1] - H[i * 3 + 1] * H[j * 3 + 0];
      };
      double cr[3];
      int pairs[3][2] = {{1, 2}, {2, 0}, {0, 1}};
      for (int a = 0; a < 3; ++a) {
        cross(pairs[a][0], pairs[a][1], cr);
        double h = vol / std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        S.nc[a] = std::max(1, std::min(64, (int)std::floor(h / (0.5 * set.cutoff))));
      }
      S.cell0 = cell0;
      cell0 += S.nc[0] * S.nc[1] * S.nc[2];
      rho_max = std::max(rho_max, d.n_atoms / vol);
      // atoms
      double sq = 0, sq2 = 0, M[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < d.n_atoms; ++i) {
        h_sysid.push_back(si);
        h_q.push_back(T(d.q[i]));
        h_rad.push_back(T(d.radius[i]));
        h_al.push_back(T(d.alpha[i]));
        h_ial.push_back(T(1.0 / d.alpha[i]));
        h_rh.push_back(T(d.lj_rmin_half[i]));
        h_se.push_back(T(d.lj_sqrt_eps[i]));
        h_mass.push_back(d.masses[i]);
        sq += d.q[i];
        sq2 += d.q[i] * d.q[i];
        double pw = 1.0;
        for (int k = 0; k < 7; ++k) { M[k] += d.lj_sqrt_eps[i] * pw; pw *= d.lj_rmin_half[i]; }
      }
      static const double binom[7] = {1, 6, 15, 20, 15, 6, 1};
      double SB = 0;
      for (int k = 0; k < 7; ++k) SB += binom[k] * M[k] * M[6 - k];
      S.tail_sb = 2.0 * SB;
      S.sum_q = sq; S.sum_q2 = sq2;
      for (int m = 0; m < d.n_mol; ++m) {
        int a0 = d.mol_start[m], a1 = d.mol_start[m + 1];
        h_molstart.push_back(atom0 + a0);
        for (int i = a0; i < a1; ++i) {
          h_molid.push_back(mol0 + m);
          h_molfirst.push_back(atom0 + a0);
          h_molend.push_back(atom0 + a1);
        }
      }
      // covalent dipoles: CSR by carrying atom, and a flat list
      std::vector<std::vector<std::pair<int, double>>> per(d.n_atoms);
      for (int c = 0; c < d.n_cov; ++c) {
        per[d.cov_i[c]].push_back({atom0 + d.cov_j[c], d.cov_c[c]});
        h_covi_flat.push_back(atom0 + d.cov_i[c]);
        h_covj_flat.push_back(atom0 + d.cov_j[c]);
        h_covc_flat.push_back(d.cov_c[c]);
      }
      for (int i = 0; i < d.n_atoms; ++i) {
        h_covstart.push_back((int)h_covj.size());
        for (auto &pr : per[i]) { h_covj.push_back(pr.first); h_covc.push_back(pr.second); }
      }
      atom0 += d.n_atoms;
      mol0 += d.n_mol;
    }
    h_molstart.push_back(atom0);
    h_covstart.push_back((int)h_covj.size());
    nt = atom0;
    nmol_total = mol0;
    ncell = cell0;
    ncov = (int)h_covi_flat.size();
    rgrid = rg;
    cgrid = cg;
    // default row capacity: the pairs in a cutoff sphere at the densest system, +25 %, + 16
    double sphere = 4.0 / 3.0 * M_PI * std::pow(set.cutoff, 3) * rho_max;
    mc_auto = std::max(32, (int)std::ceil((sphere * 1.25 + 16.0) / 32.0) * 32);
    mc = set.row_capacity > 0 ? ((set.row_capacity + 31) / 32) * 32 : mc_auto;
    rc_e = (set.elec_cutoff > 0 && set.elec_cutoff < set.cutoff && set.vdw) ? set.elec_cutoff : set.cutoff;
    split = rc_e < set.cutoff;
    if (split) {
      double se = 4.0 / 3.0 * M_PI * std::pow(rc_e, 3) * rho_max;
      mce_auto = std::max(32, (int)std::ceil((se * 1.25 + 16.0) / 32.0) * 32);
      mce = set.elec_capacity > 0 ? ((set.elec_capacity + 31) / 32) * 32 : mce_auto;
      mc = std::max(mc, mce + 32);
    } else {
      mce = mc;
    }
    // Verlet skin: cutoff + skin must stay within half of every box (minimum image)
    double halfmin = 1e300;
    for (int si = 0; si < n; ++si) {
      const double *H = systems[si].box0;
      halfmin = std::min(halfmin, 0.5 * std::min(H[0], std::min(H[4], H[8])));
    }
    skin = std::max(0.0, std::min(set.skin, halfmin - set.cutoff));
    double shell = 4.0 / 3.0 * M_PI * std::pow(set.cutoff + skin, 3) * rho_max;
    cc_auto = std::max(32, (int)std::ceil((shell * 1.25 + 32.0) / 32.0) * 32);
    cc = set.list_capacity > 0 ? ((set.list_capacity + 31) / 32) * 32 : cc_auto;
    // block maps
    std::vector<int> wbs, wba, tbs, tba;
    for (int si = 0; si < n; ++si) {
      const pgm::SysInfo &S = hsys[si];
      for (int a = 0; a < S.natom; a += pgm::WARPS_PER_BLOCK) { wbs.push_back(si); wba.push_back(S.atom0 + a); }
      for (int a = 0; a < S.natom; a += pgm::THREADS_PER_BLOCK) { tbs.push_back(si); tba.push_back(S.atom0 + a); }
    }
    nwblk = (int)wbs.size();
    ntblk = (int)tbs.size();
    wb_sys.upload(wbs); wb_atom0.upload(wba); tb_sys.upload(tbs); tb_atom0.upload(tba);
    // plane passes for the systems whose K2 = K3 mesh has a compiled plan and whose plane (two
    // regions + the twiddles) fits in a CTA's shared memory; the others run the k3 and k2 passes
    int cur_dev = 0, smem_optin = 0;
    CK(cudaGetDevice(&cur_dev));
    CK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, cur_dev));
    auto plane_ok = [&](const pgm::SysInfo &S) {
      const int L = S.K[1];
      if (L != S.K[2] || L > 128 || L % 8 != 0) return false;
      bool compiled = false;
      with_fft_len(L, [&](auto Lc) { compiled = decltype(Lc)::value != 0; });
      return compiled && plane_smem(L) <= (size_t)smem_optin;
    };
    // FFT launch groups per axis: systems with the same mesh length share one launch
    auto groups = [&](int axis, std::vector<std::unique_ptr<FftGroup>> &out) {
      std::vector<int> Ks;
      for (auto &S : hsys)
        if ((axis == 0 || !plane_ok(S)) && std::find(Ks.begin(), Ks.end(), S.K[axis]) == Ks.end()) Ks.push_back(S.K[axis]);
      for (int K : Ks) {
        std::unique_ptr<FftGroup> g(new FftGroup());
        g->K = K;
        std::vector<int> gs, gt{0};
        for (int si = 0; si < n; ++si) {
          const pgm::SysInfo &S = hsys[si];
          if (S.K[axis] != K || (axis != 0 && plane_ok(S))) continue;
          int tiles = axis == 2 ? (S.K[0] * S.K[1] + 2 * pgm::FFT_PAIRS - 1) / (2 * pgm::FFT_PAIRS)
                    : axis == 1 ? (S.K[0] * S.K3h + pgm::FFT_TILE - 1) / pgm::FFT_TILE
                                : (S.K[1] * S.K3h + pgm::FFT_TILE - 1) / pgm::FFT_TILE;
          gs.push_back(si);
          gt.push_back(gt.back() + tiles);
        }
        g->ng = (int)gs.size();
        g->ntiles = gt.back();
        g->smem = (axis == 2 ? (size_t)2 * pgm::FFT_PAIRS * K : (size_t)2 * pgm::FFT_TILE * (K + 1)) * sizeof(pgm::c2<T>) +
                  (size_t)K * sizeof(pgm::c2<T>);  // + the twiddle table
        g->sys.upload(gs);
        g->tile0.upload(gt);
        out.push_back(std::move(g));
      }
    };
    groups(2, gx);
    groups(1, gy);
    groups(0, gz);
    {
      std::vector<int> Ls;
      for (auto &S : hsys)
        if (plane_ok(S) && std::find(Ls.begin(), Ls.end(), S.K[1]) == Ls.end()) Ls.push_back(S.K[1]);
      for (int L : Ls) {
        std::unique_ptr<FftGroup> g(new FftGroup());
        g->K = L;
        std::vector<int> gs, gt{0};
        for (int si = 0; si < n; ++si) {
          if (!plane_ok(hsys[si]) || hsys[si].K[1] != L) continue;
          gs.push_back(si);
          gt.push_back(gt.back() + hsys[si].K[0]);  // one CTA per k1 plane
        }
        g->ng = (int)gs.size();
        g->ntiles = gt.back();
        g->smem = plane_smem(L);
        g->sys.upload(gs);
        g->tile0.upload(gt);
        gp.push_back(std::move(g));
      }
    }
    d_sys.upload(hsys);
    d_box.alloc(n);
    CK(cudaMemset(d_box.p, 0, sizeof(pgm::BoxInfo) * n));
    std::vector<pgm::CGSys> hcg(n);
    std::memset(hcg.data(), 0, sizeof(pgm::CGSys) * n);
    for (int si = 0; si < n; ++si) hcg[si].n3 = 3 * hsys[si].natom;
    d_cg.upload(hcg);
    d_eacc.alloc(n);
    d_status.alloc(n);
    sysid.upload(h_sysid); molid.upload(h_molid); molfirst.upload(h_molfirst); molend.upload(h_molend);
    mol_start.upload(h_molstart); cov_start.upload(h_covstart); cov_j.upload(h_covj);
    cov_i_flat.upload(h_covi_flat); cov_j_flat.upload(h_covj_flat);
    q.upload(h_q); radius.upload(h_rad); alpha.upload(h_al); ialpha.upload(h_ial); rminh.upload(h_rh); seps.upload(h_se);
    {
      std::vector<pgm::v4<T>> h_qls(nt);
      for (int k = 0; k < nt; ++k) {
        h_qls[k].x = h_q[k]; h_qls[k].y = h_rh[k]; h_qls[k].z = h_se[k]; h_qls[k].w = T(0);
      }
      qls.upload(h_qls);
    }
    mass.upload(h_mass); cov_c.upload(h_covc); cov_c_flat.upload(h_covc_flat); bmod.upload(h_bmod);
    tw.upload(h_tw);
    base.alloc(nt); frac.alloc(nt); X.alloc(nt); R.alloc(nt); Z.alloc(nt); Pv.alloc(nt); AP.alloc(nt); Bv.alloc(nt); D.alloc(nt); Fv.alloc(nt); Fpv.alloc(nt);
    pperm.alloc(nt); off.alloc(nt); dEdd.alloc(nt);
    cell_of.alloc(nt); slot_of.alloc(nt); cell_count.alloc(ncell); cell_start.alloc(ncell + 1); cell_atoms.alloc(nt); spos.alloc(nt);
    pos_ref.alloc(nt); pos4.alloc(nt); ncand.alloc(nt);
    if (sizeof(T) == 4) pos4f.alloc(nt); cand.alloc((size_t)nt * cc); nb_flag.alloc(1); nb_builds.alloc(1);
    CK(cudaMemset(cell_count.p, 0, sizeof(int) * ncell));
    CK(cudaMemset(nb_builds.p, 0, sizeof(long long)));
    { int one = 1; CK(cudaMemcpy(nb_flag.p, &one, sizeof(int), cudaMemcpyHostToDevice)); }
    rn.alloc(nt); rnsp.alloc(nt); dmax.alloc(2); dany.alloc(1); cg_done.alloc(1); dfb.alloc(1);
    if (set.iel) {  // extended-Lagrangian dipoles: Niklasson's coefficients for the order
      static const struct { int K; double kappa, a; double c[10]; } xl_table[] = {
          {0, 1.0, 0.0, {0}},
          {3, 1.69, 0.150, {-2, 3, 0, -1}},
          {4, 1.75, 0.057, {-3, 6, -2, -2, 1}},
          {5, 1.82, 0.018, {-6, 14, -8, -3, 4, -1}},
          {6, 1.84, 0.0055, {-14, 36, -27, -2, 12, -6, 1}},
          {7, 1.86, 0.0016, {-36, 99, -88, 11, 32, -25, 8, -1}},
          {8, 1.88, 0.00044, {-99, 286, -286, 78, 78, -90, 42, -10, 1}},
          {9, 1.89, 0.00012, {-286, 858, -936, 364, 168, -300, 184, -63, 12, -1}},
      };
      int row = -1;
      for (int r = 0; r < 8; ++r)
        if (xl_table[r].K == set.iel_order) row = r;
      iel_co.kappa = set.iel_custom ? set.iel_kappa : xl_table[row].kappa;
      iel_co.a = set.iel_custom ? set.iel_alpha : xl_table[row].a;
      iel_co.nc = set.iel_order == 0 ? 1 : set.iel_order + 1;
      for (int k = 0; k < iel_co.nc; ++k) iel_co.c[k] = xl_table[row].c[k];
      iel_co.K1 = pgm_iel_len(set.iel_order);
      iel_co.zscf = set.iel == 1;
      iel_len = iel_co.K1;
      iel_warmup = std::max(set.iel_order, 2) + 1;
      iel_shadow = set.iel == 1 && !set.iel_no_shadow;
      Dl.alloc(nt);
      CK(cudaMemset(Dl.p, 0, sizeof(pgm::v4<T>) * nt));
      if (iel_shadow) {
        Phi2.alloc(rgrid);
        d_eacc2.alloc(nsys);
      }
    }
    CK(cudaMemset(cg_done.p, 0, sizeof(unsigned)));
    if (split) rnv.alloc(nt);
    alloc_rows();
    Q.alloc(rgrid); Phi.alloc(rgrid); Ginf.alloc(cgrid); C.alloc(cgrid);
    CK(cudaMemset(Q.p, 0, sizeof(T) * rgrid));
    mu_tmp.alloc((size_t)3 * nt); forces_tmp.alloc((size_t)3 * nt); energy_tmp.alloc((size_t)3 * n);
    nn_w.alloc(pgmnn::NN_NPARAM); nn_wb.alloc(pgmnn::NN_WB_ELEMS); nn_inv.alloc((size_t)nt * pgmnn::NN_IN); nn_vec.alloc((size_t)nt * pgmnn::NN_CH * 3);
    nn_mu.alloc((size_t)nt * 3); nn_chan.alloc((size_t)nt * pgm::NN_CHAN); nn_bl.alloc(nt); nn_valid.alloc(1);
    if (set.predictor == 5) ensure_graph();
    if (set.local_niter > 0) {
      const size_t ns = (size_t)nt * SH_MAX;
      sh_n.alloc(nt); c_k.alloc(ns);
      c_x.alloc(ns); c_y.alloc(ns); c_z.alloc(ns); c_g1.alloc(ns); c_g2.alloc(ns);
      LRR.alloc(nt); LZZ.alloc(nt); LP0.alloc(nt); LP1.alloc(nt); DRv.alloc(nt);
      CK(cudaMemset(sh_n.p, 0, sizeof(int) * nt));
    }
    CK(cudaMemset(nn_valid.p, 0, sizeof(int)));
    CK(cudaMallocHost(&h_any, sizeof(int)));
    CK(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&aux_b, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_fork_b, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_join_b, cudaEventDisableTiming));
    int prio_lo = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    {
      int d = 0;
      CK(cudaGetDevice(&d));
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, d));
    }
    CK(cudaStreamCreateWithPriority(&nn_st, cudaStreamNonBlocking, prio_hi));
    CK(cudaEventCreateWithFlags(&ev_nn_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_nn_join, cudaEventDisableTiming));
    set_smem();
  }

  void alloc_rows() {
    ++generation;
    size_t m = (size_t)nt * mc;
    rk.alloc(m); rx.alloc(m); ry.alloc(m); rz.alloc(m); rg0.alloc(m); rg1.alloc(m); rg2.alloc(m); rg3.alloc(m);
  }

  static size_t plane_smem(int L) { return (size_t)(2 * pgm::plane_region(L) + L) * sizeof(pgm::c2<T>); }

  // Plane-pass lengths: the compiled plans up to 128 (a 192 plane does not fit in shared memory).
  template <typename F>
  static void with_plane_len(int L, F &&f) {
    with_fft_len(L, [&](auto Lc) {
      constexpr int Lv = decltype(Lc)::value;
      if constexpr (Lv > 0 && Lv <= 128) f(Lc);
    });
  }

  template <typename K>
  void smem_attr(K kern, size_t bytes) {
    if (bytes > 48 * 1024) CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  }

  void set_smem() {
    for (auto &g : gp)
      with_plane_len(g->K, [&](auto Lc) {
        constexpr int L = decltype(Lc)::value;
        smem_attr(pgm::k_fft_plane_fwd<T, L>, g->smem);
        smem_attr(pgm::k_fft_plane_inv<T, L>, g->smem);
      });
    for (auto &g : gx)
      with_fft_len(g->K, [&](auto Lc) {
        constexpr int L = decltype(Lc)::value;
        smem_attr(pgm::k_fft_x_fwd<T, L>, g->smem);
        smem_attr(pgm::k_fft_x_inv<T, L>, g->smem);
      });
    for (auto &g : gy)
      with_fft_len(g->K, [&](auto Lc) {
        constexpr int L = decltype(Lc)::value;
        smem_attr(pgm::k_fft_y<T, L>, g->smem);
      });
    for (auto &g : gz)
      with_fft_len(g->K, [&](auto Lc) {
        constexpr int L = decltype(Lc)::value;
        smem_attr(pgm::k_fft_z_conv<T, L, false>, g->smem);
        smem_attr(pgm::k_fft_z_conv<T, L, true>, g->smem);
      });
  }

  // The forward plane passes (k3 + k2 per k1 plane) of the systems that have them.
  void plane_fwd(cudaStream_t st, pgm::Dev<T> &a, int act) {
    for (auto &g : gp)
      with_plane_len(g->K, [&](auto Lc) {
        launch_pdl(pgm::k_fft_plane_fwd<T, decltype(Lc)::value>, g->ntiles, pgm::PLANE_THREADS, g->smem, st, a,
                   (const int *)g->sys.p, (const int *)g->tile0.p, g->ng, act);
      });
  }

  // The passes of one reciprocal-space convolution: r2c (k3) and k2 -- one plane pass where the
  // mesh has it --, k1 with G, k2 and c2r (k3).
  void fft_chain(cudaStream_t st, pgm::Dev<T> &a, int act, bool energy) {
    plane_fwd(st, a, act);
    for (auto &g : gx)
      with_fft_len(g->K, [&](auto Lc) {
        launch_pdl(pgm::k_fft_x_fwd<T, decltype(Lc)::value>, g->ntiles, pgm::FFT_THREADS, g->smem, st, a, (const int *)g->sys.p,
                   (const int *)g->tile0.p, g->ng, act);
      });
    for (auto &g : gy)
      with_fft_len(g->K, [&](auto Lc) {
        launch_pdl(pgm::k_fft_y<T, decltype(Lc)::value>, g->ntiles, pgm::FFT_THREADS, g->smem, st, a, (const int *)g->sys.p,
                   (const int *)g->tile0.p, g->ng, act, -1);
      });
    for (auto &g : gz)
      with_fft_len(g->K, [&](auto Lc) {
        if (energy)
          launch_pdl(pgm::k_fft_z_conv<T, decltype(Lc)::value, true>, g->ntiles, pgm::FFT_THREADS, g->smem, st, a,
                     (const int *)g->sys.p, (const int *)g->tile0.p, g->ng, act);
        else
          launch_pdl(pgm::k_fft_z_conv<T, decltype(Lc)::value, false>, g->ntiles, pgm::FFT_THREADS, g->smem, st, a,
                     (const int *)g->sys.p, (const int *)g->tile0.p, g->ng, act);
      });
    for (auto &g : gy)
      with_fft_len(g->K, [&](auto Lc) {
        launch_pdl(pgm::k_fft_y<T, decltype(Lc)::value>, g->ntiles, pgm::FFT_THREADS, g->smem, st, a, (const int *)g->sys.p,
                   (const int *)g->tile0.p, g->ng, act, +1);
      });
    for (auto &g : gx)
      with_fft_len(g->K, [&](auto Lc) {
        launch_pdl(pgm::k_fft_x_inv<T, decltype(Lc)::value>, g->ntiles, pgm::FFT_THREADS, g->smem, st, a, (const int *)g->sys.p,
                   (const int *)g->tile0.p, g->ng, act);
      });
    for (auto &g : gp)
      with_plane_len(g->K, [&](auto Lc) {
        launch_pdl(pgm::k_fft_plane_inv<T, decltype(Lc)::value>, g->ntiles, pgm::PLANE_THREADS, g->smem, st, a,
                   (const int *)g->sys.p, (const int *)g->tile0.p, g->ng, act);
      });
  }

  // ---------------------------------------------------------------- autotuner
  // The tuned kernels: the CG matvec's row stream k_rowfield (lanes per row 32 / 16 / 8: how a
  // neighbour row is split over a warp) and the force pass k_forces (at least 2 / 3 / 4 blocks of
  // 256 threads per SM: registers against resident warps).
  // beside: forked beside the FFT chain, where the tuned grid limit (tune.rowfield_grid blocks per
  // SM, at the highest priority) applies; 0 or not beside: one block per 8 rows.
  template <bool WITH_Q, int ACT>
  void rowfield(cudaStream_t st, pgm::Dev<T> &a, const pgm::v4<T> *vin, pgm::v4<T> *out, bool pdl, int lpr = 0,
                bool beside = false, int grid_per_sm = -1) {
    const int g = grid_per_sm >= 0 ? grid_per_sm : tune.rowfield_grid;
    auto go = [&](auto L) {
      constexpr int LPR = decltype(L)::value;
      if (pdl) {
        launch_pdl(pgm::k_rowfield<T, WITH_Q, ACT, LPR>, nwblk, 8 * LPR, 0, st, a, vin, out, nwblk);
      } else if (beside && g > 0) {  // variant g: 4 g blocks per SM, walking the rows at the grid's stride
        launch_prio(pgm::k_rowfield<T, WITH_Q, ACT, LPR>, (unsigned)std::min(nwblk, 4 * g * nsm), 8 * LPR, 0, st, prio_hi,
                    a, vin, out, nwblk);
      } else {
        pgm::k_rowfield<T, WITH_Q, ACT, LPR><<<nwblk, 8 * LPR, 0, st>>>(a, vin, out, nwblk);
        check_launch();
      }
    };
    const int l = lpr ? lpr : tune.rowfield_lanes;
    if (l == 16) go(std::integral_constant<int, 16>{});
    else if (l == 8) go(std::integral_constant<int, 8>{});
    else go(std::integral_constant<int, 32>{});
  }
  void forces_pass(cudaStream_t st, pgm::Dev<T> &a, const double *mu, bool pdl, int minb = 0, bool shadow = false) {
    auto go = [&](auto B) {
      constexpr int MINB = decltype(B)::value;
      if (shadow) {  // iEL/0-SCF: the shadow potential's energy and forces
        launch_pdl(pgm::k_forces<T, P, MINB, true, FORCES_LPA>, nwblk, 8 * FORCES_LPA, 0, st, a, mu);
      } else if (pdl) {
        launch_pdl(pgm::k_forces<T, P, MINB, false, FORCES_LPA>, nwblk, 8 * FORCES_LPA, 0, st, a, mu);
      } else {
        pgm::k_forces<T, P, MINB, false, FORCES_LPA><<<nwblk, 8 * FORCES_LPA, 0, st>>>(a, mu);
        check_launch();
      }
    };
    const int b = minb ? minb : tune.forces_blocks_per_sm;
    if (b == 2) go(std::integral_constant<int, 2>{});
    else if (b == 4) go(std::integral_constant<int, 4>{});
    else go(std::integral_constant<int, 3>{});
  }
  void set_tuning(int lanes, int blocks, int early, int grid) override {
    ++generation;  // captured steps hold the old variants
    tune_fixed = lanes > 0 || blocks > 0 || early >= 0 || grid >= 0;
    if (lanes > 0) tune.rowfield_lanes = lanes;
    if (blocks > 0) tune.forces_blocks_per_sm = blocks;
    if (early >= 0) tune.sweep_early = early;
    if (grid >= 0) tune.rowfield_grid = grid;
    if (!tune_fixed) tune.tuned = 0;  // autotune again at the next direct step
  }
  PgmTuning tuning() const override { return tune; }
  // Times every variant on this handle's rows (the last step's geometry; CUDA events on st, a
  // warm-up launch and the mean of 10) and keeps the fastest of each kernel.  Writes only scratch
  // buffers: the last call's outputs are untouched.
  void autotune(cudaStream_t st) override {
    const TuneKey key{(int)sizeof(T), P, nt, mc, rgrid};
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tune_cache.find(key);
      if (it != g_tune_cache.end()) {
        tune = it->second;
        tune.from_cache = 1;
        ++generation;
        return;
      }
    }
    pgm::Dev<T> a = dev(nullptr, nullptr, 0, forces_tmp.p, d_status.p);
    a.pos = last_pos;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const long long l0 = launches;
    auto time = [&](auto &&launch) {
      launch();
      CK(cudaEventRecord(e0, st));
      for (int r = 0; r < 10; ++r) launch();
      CK(cudaEventRecord(e1, st));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      return ms / 10.0;
    };
    const int lanes[3] = {32, 16, 8}, blocks[3] = {2, 3, 4};
    int bl = 0, bb = 0;
    for (int v = 0; v < 3; ++v) {
      tune.rowfield_ms[v] = time([&] { rowfield<false, 0>(st, a, X.p, Fv.p, false, lanes[v]); });
      tune.forces_ms[v] = time([&] { forces_pass(st, a, nullptr, false, blocks[v]); });
      if (tune.rowfield_ms[v] < tune.rowfield_ms[bl]) bl = v;
      if (tune.forces_ms[v] < tune.forces_ms[bb]) bb = v;
    }
    tune.rowfield_lanes = lanes[bl];
    // the CG direction's sweep (spread with the update of p, FFT chain, row field, gather) with the
    // row field forked after the spread or at the start of the sweep (on z)
    if (overlap) {
      for (int v = 0; v < 2; ++v) {
        tune.sweep_early = v;
        tune.sweep_ms[v] = time([&] { sweep<false, true, 0, 1>(st, a, Pv.p, AP.p); });
      }
      tune.sweep_early = tune.sweep_ms[1] < tune.sweep_ms[0] ? 1 : 0;
      // the row field beside the FFT chain on all SMs, or on 4 or 8 blocks per SM at the highest
      // priority (the FFT passes fill the rest of each SM)
      int bg = 0;
      for (int v = 0; v < 3; ++v) {
        tune.rowfield_grid = v;
        tune.grid_ms[v] = time([&] { sweep<false, true, 0, 1>(st, a, Pv.p, AP.p); });
        if (tune.grid_ms[v] < tune.grid_ms[bg]) bg = v;
      }
      tune.rowfield_grid = bg;
    }
    CK(cudaMemsetAsync(Q.p, 0, sizeof(T) * rgrid, st));  // leave the spread grid cleared
    launches = l0;
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    tune.rowfield_lanes = lanes[bl];
    tune.forces_blocks_per_sm = blocks[bb];
    tune.tuned = 1;
    tune.from_cache = 0;
    ++generation;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = tune;
  }

  void set_nn_fallback(double factor) override {
    ++generation;  // a captured step holds the fallback node only when the check is on
    nn_fb_factor = factor;
  }
  void nn_fallback_stats(long long *fallbacks, double *ref_err) override {
    std::vector<pgm::CGSys> h(nsys);
    CK(cudaMemcpy(h.data(), d_cg.p, sizeof(pgm::CGSys) * nsys, cudaMemcpyDeviceToHost));
    for (int k = 0; k < nsys; ++k) {
      if (fallbacks) fallbacks[k] = h[k].fallbacks;
      if (ref_err) ref_err[k] = h[k].ref_n > 0 ? h[k].ref_err : -1.0;
    }
  }

  // The message-passing model (pgm_mpnn.cu) on the same features and on the graph the row build
  // writes; it replaces the MLP as the learned guess until set_nn or set_mpnn(null).
  // The graph's edge list (allocated with predictor 5, else when a model is installed or the
  // features are asked for).
  void ensure_graph() {
    if (!nn_e4.p) { nn_e4.alloc((size_t)nt * NN_EMAX); nn_g.alloc((size_t)nt * NN_EMAX); nn_ne.alloc(nt); }
  }

  void set_mpnn(const float *w, int nparam, float sigma, float rg) override {
    ++generation;
    ensure_graph();
    mp_on = w != nullptr;
    nn_on = mp_on;
    if (w) {
      mp_w.alloc(nparam);
      CK(cudaMemcpy(mp_w.p, w, sizeof(float) * nparam, cudaMemcpyDeviceToDevice));
      mp_work.alloc(pgmmp_engine::work_bytes(nt));
      CK(pgmmp_engine::set_weights(mp_w.p, mp_work.p, nt, 0));
      CK(cudaDeviceSynchronize());
    }
    CK(cudaMemset(nn_valid.p, 0, sizeof(int)));
    nn_sigma = sigma;
    nn_rg = rg;
  }
  // The graph of the last step (edges (x, y, z, partner) per atom, up to emax, and their counts).
  void nn_graph(cudaStream_t st, float4 *edges, int *counts, int emax) override {
    if (!nn_e4.p) throw CudaError{"the graph is kept only with predictor 5 (learned guess)"};
    CK(cudaMemcpy2DAsync(edges, sizeof(float4) * emax, nn_e4.p, sizeof(float4) * NN_EMAX, sizeof(float4) * std::min(emax, NN_EMAX),
                         nt, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(counts, nn_ne.p, sizeof(int) * nt, cudaMemcpyDeviceToDevice, st));
  }

  void set_nn(const float *w, float sigma, float rg) override {
    ensure_graph();
    ++generation;  // a captured step depends on whether a model is set, and on sigma and rg
    mp_on = false;
    nn_on = w != nullptr;
    if (w) {
      CK(cudaMemcpy(nn_w.p, w, sizeof(float) * pgmnn::NN_NPARAM, cudaMemcpyDeviceToDevice));
      CK(pgmnn::nn_weights_bf16(nn_w.p, nn_wb.p, 0));  // the matrices as the inference kernel reads them
      CK(cudaDeviceSynchronize());
    }
    CK(cudaMemset(nn_valid.p, 0, sizeof(int)));
    nn_sigma = sigma;
    nn_rg = rg;
  }

  // The model's inputs at a geometry (the row build wrote the graph's edges): the graph's permanent
  // field (written to bl_out; its change from bl_prev, when given, is a channel) and the history
  // channels.
  void nn_inputs(cudaStream_t st, pgm::Dev<T> &a, const double *hist, const float4 *bl_prev, const int *valid, float4 *bl_out,
                 float *inv, float *vec, int *set_valid) {
    if (!a.nn_e4) throw CudaError{"the learned guess's graph list is not allocated"};
    launch_prio(pgm::k_nn_chan<T, CHAN_LPA>, nwblk, 8 * CHAN_LPA, 0, st, prio_hi, a, hist, bl_prev, valid, nn_rg, bl_out, nn_chan.p);
    launch_prio(pgm::k_nn_features<T>, nwblk, 256, 0, st, prio_hi, a, (const float *)nn_chan.p, nn_sigma, nn_rg, inv, vec,
                set_valid);
  }

  void nn_features(cudaStream_t st, const double *pos, const double *box, const double *hist, const float *bl_prev,
                   float *bl_out, float *inv, float *vec) override {
    launches = 0;
    ensure_graph();
    CK(cudaMemsetAsync(d_status.p, 0, sizeof(unsigned) * nsys, st));
    pgm::Dev<T> a = dev(pos, nullptr, 0, forces_tmp.p, d_status.p);
    prepare(st, a, box);
    nn_inputs(st, a, hist, reinterpret_cast<const float4 *>(bl_prev), nullptr, reinterpret_cast<float4 *>(bl_out), inv, vec,
              nullptr);
  }

  void set_capacity(int c) override {
    int want = c > 0 ? ((c + 31) / 32) * 32 : mc_auto;
    if (split) want = std::max(want, mce + 32);
    if (want != mc) {
      mc = want;
      if (!split) mce = mc;
      alloc_rows();
    }
  }
  int capacity() const override { return mc; }
  bool set_elec_capacity(int c) override {
    if (!split) return false;
    mce = c > 0 ? ((c + 31) / 32) * 32 : mce_auto;
    ++generation;
    if (mc < mce + 32) {
      mc = mce + 32;
      alloc_rows();
    }
    return true;
  }
  int elec_capacity() const override { return mce; }
  int max_vdw_count() override {
    int v[2] = {0, 0};
    CK(cudaMemcpy(v, dmax.p, sizeof(v), cudaMemcpyDeviceToHost));
    return v[1];
  }
  long long launches_per_iteration() const override { return per_iter; }

  // Average duration [ms] of one launch of a kernel of the last step, re-run `reps` times on the
  // state that step left (rows, vectors, grids): 0 the CG matvec (rows + PME gather), 1 the spread,
  // 2 the FFT/convolution chain, 3 the energy/force pass, 4 the row build.
  bool has_hist() const override { return last_hist != nullptr; }
  double profile(cudaStream_t st, int which, int reps) override {
    pgm::Dev<T> a = dev(nullptr, nullptr, 0, forces_tmp.p, d_status.p);
    a.pos = last_pos;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto one = [&]() {
      if (which == 0) pgm::k_rowmat<T, P, false, 1, 0><<<nwblk, 256, 0, st>>>(a, Pv.p, AP.p);
      else if (which == 1) pgm::k_spread<T, P, false, false, 0, SPREAD_LPA><<<nwblk, 8 * SPREAD_LPA, 0, st>>>(a, Pv.p);
      else if (which == 2) {
        fft_chain(st, a, 0, false);
      } else if (which == 3) forces_pass(st, a, nullptr, false);
      else if (which == 4) {
        pgm::k_rows<T, ROWS_LPA, ROWS_TWO_PHASE><<<nwblk, 8 * ROWS_LPA, 0, st>>>(a);
      }
      else if (which == 5 || which == 6) {  // the first FFT pass (plane or k3), after the spread with 6
        if (which == 6) pgm::k_spread<T, P, false, false, 0, SPREAD_LPA><<<nwblk, 8 * SPREAD_LPA, 0, st>>>(a, Pv.p);
        plane_fwd(st, a, 0);
        for (auto &g : gx)
          with_fft_len(g->K, [&](auto Lc) {
            pgm::k_fft_x_fwd<T, decltype(Lc)::value><<<g->ntiles, pgm::FFT_THREADS, g->smem, st>>>(a, g->sys.p, g->tile0.p, g->ng, 0);
          });
      } else if (which == 7) rowfield<false, 0>(st, a, Pv.p, Fv.p, false);
      else if (which == 8) pgm::k_rowmat<T, P, false, 1, 0, false, false, GATHER_LPA><<<nwblk, 8 * GATHER_LPA, 0, st>>>(a, Pv.p, AP.p);
      else if (which == 9) {  // a whole operator sweep with the row/PME overlap
        sweep<false, false, 0, 1>(st, a, Pv.p, AP.p);
      } else if (which == 10) {  // the learned guess's channel pass (rewrites the same graph field)
        pgm::k_nn_chan<T, CHAN_LPA><<<nwblk, 8 * CHAN_LPA, 0, st>>>(a, last_hist, nn_bl.p, nullptr, nn_rg, nn_bl.p, nn_chan.p);
      } else if (which == 11) {
        pgm::k_nn_features<T><<<nwblk, 256, 0, st>>>(a, nn_chan.p, nn_sigma, nn_rg, nn_inv.p, nn_vec.p, nullptr);
      } else {  // 12: the model
        CK(mp_on ? pgmmp_engine::predict(mp_w.p, mp_work.p, nn_inv.p, nn_vec.p, nn_e4.p, nn_ne.p, NN_EMAX, nt, nn_sigma, nn_rg,
                                         nn_mu.p, st, 0)
                 : pgmnn::nn_predict_launch(nn_w.p, nn_wb.p, nn_inv.p, nn_vec.p, nt, nn_mu.p, st));
      }
    };
    long long l0 = launches;
    one();  // warm-up
    CK(cudaGetLastError());
    CK(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) one();
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    CK(cudaMemsetAsync(Q.p, 0, sizeof(T) * rgrid, st));  // leave the spread grid cleared
    launches = l0;
    CK(cudaEventDestroy(e0));
    CK(cudaEventDestroy(e1));
    CK(cudaGetLastError());
    return ms / reps;
  }

  // In-cutoff pairs of the last row build (sum over rows).
  long long row_pairs() override {
    std::vector<int> h(nt);
    CK(cudaMemcpy(h.data(), rn.p, sizeof(int) * nt, cudaMemcpyDeviceToHost));
    long long t = 0;
    for (int v : h) t += std::min(v, mce);
    return t;
  }
  int max_count() override {
    int v = 0;
    CK(cudaMemcpy(&v, dmax.p, sizeof(int), cudaMemcpyDeviceToHost));
    return v;
  }

  void check_launch() {
    ++launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError{std::string("kernel launch: ") + cudaGetErrorString(e)};
  }

  int grid1(int n, int b = 256) { return (n + b - 1) / b; }

  // Launch with programmatic stream serialization: the kernel (which begins with pdl_enter()) is
  // scheduled while its predecessor drains, so the per-kernel launch gap of the CG loop overlaps
  // the previous kernel's tail; after a non-kernel node the attribute has no effect.
  template <typename... KArgs, typename... Args>
  void launch_pdl(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k, args...));
    ++launches;
  }

  // A launch at scheduling priority prio (a node attribute when captured: the block scheduler
  // dispatches its blocks ahead of those of concurrent lower-priority kernels).
  template <typename... KArgs, typename... Args>
  void launch_prio(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st, int prio, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributePriority;
    at[0].val.priority = prio;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k, args...));
    ++launches;
  }

  // Geometry of a step: box, fractional coordinates and permanent dipoles, molecular offsets,
  // cell list, rows, influence function.
  // The learned guess's inputs and prediction for this step's graph: forked onto nn_st after the
  // row build, beside the influence function and the solve's set-up; solve() joins it.
  void nn_fork(cudaStream_t st, pgm::Dev<T> &a, const double *hist) {
    CK(cudaEventRecord(ev_nn_fork, st));
    CK(cudaStreamWaitEvent(nn_st, ev_nn_fork, 0));
    nn_inputs(nn_st, a, hist, nn_bl.p, nn_valid.p, nn_bl.p, nn_inv.p, nn_vec.p, nn_valid.p);
    cudaError_t e = mp_on ? pgmmp_engine::predict(mp_w.p, mp_work.p, nn_inv.p, nn_vec.p, nn_e4.p, nn_ne.p, NN_EMAX, nt, nn_sigma,
                                                  nn_rg, nn_mu.p, nn_st, prio_hi)
                          : pgmnn::nn_predict_launch(nn_w.p, nn_wb.p, nn_inv.p, nn_vec.p, nt, nn_mu.p, nn_st, prio_hi);
    if (e != cudaSuccess) throw CudaError{std::string("nn_predict: ") + cudaGetErrorString(e)};
    ++launches;
    CK(cudaEventRecord(ev_nn_join, nn_st));
    nn_forked = true;
  }

  void prepare(cudaStream_t st, pgm::Dev<T> &a, const double *boxes, const double *nn_hist = nullptr) {
    launch_pdl(pgm::k_box<T>, grid1(nsys, 64), 64, 0, st, a, boxes);
    launch_pdl(pgm::k_prep<T>, grid1(nt), 256, 0, st, a);
    launch_pdl(pgm::k_mol<T>, grid1(nmol_total), 256, 0, st, a);
    if (!a.idx) {  // the Verlet candidate list, rebuilt on the device when the flag is up
      launch_pdl(pgm::k_cell_assign<T>, grid1(nt), 256, 0, st, a);
      launch_pdl(pgm::k_scan_cells, 1, 1024, 0, st, (const int *)cell_count.p, cell_start.p, ncell, (const int *)nb_flag.p);
      launch_pdl(pgm::k_scatter<T>, grid1(nt), 256, 0, st, a);
      launch_pdl(pgm::k_cand<T>, nwblk, 256, 0, st, a);
      launch_pdl(pgm::k_nb_finish, std::max(1, std::min(1024, grid1(ncell))), 256, 0, st, cell_count.p, ncell, nb_flag.p,
                 nb_builds.p);
      launch_pdl(pgm::k_nb_lower, 1, 1, 0, st, nb_flag.p, nb_builds.p);
    }
    launch_pdl(pgm::k_rows<T, ROWS_LPA, ROWS_TWO_PHASE>, nwblk, 8 * ROWS_LPA, 0, st, a);
    if (nn_hist) nn_fork(st, a, nn_hist);
    launch_pdl(pgm::k_influence<T>, (int)std::min<long long>(4096, (cgrid + 255) / 256), 256, 0, st, a, (long long)cgrid);
  }

  void set_list_capacity(int c) override {
    int want = c > 0 ? ((c + 31) / 32) * 32 : cc_auto;
    if (want != cc) {
      cc = want;
      cand.alloc((size_t)nt * cc);
      ++generation;
    }
    int one = 1;
    CK(cudaMemcpy(nb_flag.p, &one, sizeof(int), cudaMemcpyHostToDevice));
  }
  int list_capacity() const override { return cc; }
  long long list_rebuilds() override {
    long long v = 0;
    CK(cudaMemcpy(&v, nb_builds.p, sizeof(v), cudaMemcpyDeviceToHost));
    return v;
  }

  // Reciprocal-space potential phi of the grid spread from `vin` (with charges if WITH_Q).
  template <bool WITH_Q, bool UPDATE_P, int ACT, bool ENERGY>
  void pme(cudaStream_t st, pgm::Dev<T> &a, const pgm::v4<T> *vin) {
    // Q is zero here: cleared at creation and, after every spread, by the forward k2 FFT pass
    launch_pdl(pgm::k_spread<T, P, WITH_Q, UPDATE_P, ACT, SPREAD_LPA>, nwblk, 8 * SPREAD_LPA, 0, st, a, vin);
    fft_chain(st, a, ACT, ENERGY);
  }

  // One field sweep of the dipoles vin (charges with WITH_Q): the spread (after the CG direction
  // update with UPDATE_P), then the row field on a second stream beside the FFT chain, joined by
  // the PME gather that assembles MODE 0 (field) or 1 (operator, with p.Ap) into out.
  template <bool WITH_Q, bool UPDATE_P, int ACT, int MODE>
  void sweep(cudaStream_t st, pgm::Dev<T> &a, const pgm::v4<T> *vin, pgm::v4<T> *out) {
    if (!overlap) {
      // one stream: the row field runs between the spread and the first FFT pass, while the L2
      // still processes the spread's atomic adds, then the FFTs and the PME gather
      // Q is zero here: cleared at creation and, after every spread, by the forward k2 FFT pass
      pgm::k_spread<T, P, WITH_Q, UPDATE_P, ACT, SPREAD_LPA><<<nwblk, 8 * SPREAD_LPA, 0, st>>>(a, vin); check_launch();
      const pgm::v4<T> *dv = UPDATE_P ? Pv.p : vin;
      rowfield<WITH_Q, ACT>(st, a, dv, Fv.p, true);
      fft_chain(st, a, ACT, false);
      launch_pdl(pgm::k_rowmat<T, P, WITH_Q, MODE, ACT, false, false, GATHER_LPA>, nwblk, 8 * GATHER_LPA, 0, st, a, dv, out);
      return;
    }
    // the loop body is captured as a sequence of its own: it forks to its own stream
    cudaStream_t ax = in_body ? aux_b : aux;
    cudaEvent_t ef = in_body ? ev_fork_b : ev_fork, ej = in_body ? ev_join_b : ev_join;
    if (tune.sweep_early) {
      // the row field starts with the sweep, beside the spread and the FFT chain; for a CG
      // direction it takes z (the rows of p = z + beta p_prev are combined in the gather)
      CK(cudaEventRecord(ef, st));
      CK(cudaStreamWaitEvent(ax, ef, 0));
      rowfield<WITH_Q, ACT>(ax, a, UPDATE_P ? Z.p : vin, Fv.p, false, 0, true);
      CK(cudaEventRecord(ej, ax));
      launch_pdl(pgm::k_spread<T, P, WITH_Q, UPDATE_P, ACT, SPREAD_LPA>, nwblk, 8 * SPREAD_LPA, 0, st, a, vin);
      fft_chain(st, a, ACT, false);
      CK(cudaStreamWaitEvent(st, ej, 0));
      launch_pdl(pgm::k_rowmat<T, P, WITH_Q, MODE, ACT, false, UPDATE_P, GATHER_LPA>, nwblk, 8 * GATHER_LPA, 0, st, a, vin, out);
      return;
    }
    launch_pdl(pgm::k_spread<T, P, WITH_Q, UPDATE_P, ACT, SPREAD_LPA>, nwblk, 8 * SPREAD_LPA, 0, st, a, vin);
    CK(cudaEventRecord(ef, st));
    CK(cudaStreamWaitEvent(ax, ef, 0));
    rowfield<WITH_Q, ACT>(ax, a, vin, Fv.p, false, 0, true);
    CK(cudaEventRecord(ej, ax));
    fft_chain(st, a, ACT, false);
    CK(cudaStreamWaitEvent(st, ej, 0));
    // a programmatic dependent of the last FFT pass; griddepcontrol.wait also covers the joined row field
    launch_pdl(pgm::k_rowmat<T, P, WITH_Q, MODE, ACT, false, false, GATHER_LPA>, nwblk, 8 * GATHER_LPA, 0, st, a, vin, out);
  }

  // The local preconditioner's chain z = M^-1 r (k_lp_start, then per inner iteration k_lp_ap and
  // k_lp_step), for the systems ACT selects (0 all, 1 iterating, 3 falling back); MODE 0 ends with
  // p = z and r.z (a start), MODE 1 with the outer CG's check (an iteration).
  template <int ACT, int MODE>
  void local_precond(cudaStream_t st, pgm::Dev<T> &a, cudaGraphConditionalHandle cond, int use_cond) {
    const int L = set.local_niter;
    launch_pdl(pgm::k_lp_start<T, ACT>, ntblk, 256, 0, st, a);
    for (int j = 1; j <= L; ++j) {
      pgm::v4<T> *cur = (j & 1) ? LP0.p : LP1.p, *prev = (j & 1) ? LP1.p : LP0.p;
      if (j == 1) launch_pdl(pgm::k_lp_ap<T, ACT, true>, ntblk, 256, 0, st, a, (const pgm::v4<T> *)prev, cur);
      else launch_pdl(pgm::k_lp_ap<T, ACT, false>, ntblk, 256, 0, st, a, (const pgm::v4<T> *)prev, cur);
      if (j < L)
        launch_pdl(pgm::k_lp_step<T, ACT, false, MODE>, ntblk, 256, 0, st, a, (const pgm::v4<T> *)cur, nsys, set.dipole_tol,
                   set.max_iter, dany.p, cond, use_cond, cg_done.p);
      else
        launch_pdl(pgm::k_lp_step<T, ACT, true, MODE>, ntblk, 256, 0, st, a, (const pgm::v4<T> *)cur, nsys, set.dipole_tol,
                   set.max_iter, dany.p, cond, use_cond, cg_done.p);
    }
  }

  // One CG iteration: p = z + beta p spread, FFTs, A p with p.Ap, update, per-system check (with
  // the local preconditioner: the update, then its chain, whose last kernel checks).
  void iteration(cudaStream_t st, pgm::Dev<T> &a, cudaGraphConditionalHandle cond, int use_cond) {
    sweep<false, true, 1, 1>(st, a, Pv.p, AP.p);
    if (set.local_niter > 0) {
      launch_pdl(pgm::k_cg_update_r<T>, ntblk, 256, 0, st, a);
      local_precond<1, 1>(st, a, cond, use_cond);
      return;
    }
    launch_pdl(pgm::k_cg_update_check<T>, ntblk, 256, 0, st, a, nsys, set.dipole_tol, set.max_iter, dany.p, cond, use_cond,
               cg_done.p);
  }

  // Adds a conditional node (IF or WHILE on `cond`) after the capture's current dependencies of
  // st, captures body(stream) into the node's body graph (on the side stream, with the sweep's
  // fork on aux_b), and makes the node the capture's new dependency.
  template <typename F>
  void conditional_node(cudaStream_t st, cudaGraphConditionalHandle cond, cudaGraphConditionalNodeType type, F &&body) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    unsigned long long id;
    CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = cond;
    np.conditional.type = type;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, nd, &np));
    cudaGraph_t bg = np.conditional.phGraph_out[0];
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    if (!side) CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    CK(cudaStreamBeginCaptureToGraph(side, bg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    in_body = true;
    try {
      body(side);
    } catch (...) {
      in_body = false;
      cudaGraph_t junk;
      cudaStreamEndCapture(side, &junk);
      throw;
    }
    in_body = false;
    CK(cudaStreamEndCapture(side, &bg));
  }

  bool any_active(cudaStream_t st) {
    CK(cudaMemcpyAsync(h_any, dany.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return *h_any != 0;
  }

  // The induced-dipole solve (forcefield.py:1917-2008 and 1714-1821).  mode 0: predictor start
  // and history push (compute); mode 1: plain start from ind->mu, no push (energy).
  void solve(cudaStream_t st, pgm::Dev<T> &a, PgmInduction *ind, int mode, double *mu_out, int32_t *iters, double *resid) {
    // predictor 5 ("nn"): the mu4 extrapolation plus the learned correction, for systems with four
    // steps of history, with mu4's (fused) start; without a model, mu4.  Predictor 1: the previous
    // step's dipoles.
    const bool use_nn = mode == 0 && set.predictor == 5 && nn_on;
    const int pred = set.predictor == 5 ? 4 : set.predictor;
    const int K = pred == 4 ? 4 : (pred == 3 ? 3 : (pred == 1 ? 1 : 0));
    const double c4[4] = {4.0, -6.0, 4.0, -1.0}, c3[4] = {3.0, -3.0, 1.0, 0.0}, c1[4] = {1.0, 0, 0, 0}, c0[4] = {0, 0, 0, 0};
    const double *cc = K == 4 ? c4 : (K == 3 ? c3 : (K == 1 ? c1 : c0));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    const bool captured = cs == cudaStreamCaptureStatusActive;
    // captured: the plain start's second sweep sits in a conditional IF node whose condition
    // k_cg_setup raises when some system takes the plain start (else the node's kernels are skipped)
    // the learned guess's check: its start residual against the record of the extrapolation's
    // (k_cg_begin); a fallback restarts those systems from x4 with one operator sweep, captured in
    // a conditional IF node that runs only when some system falls back
    const bool check_nn = use_nn && nn_fb_factor > 0.0;
    cudaGraphConditionalHandle cond2 = 0, condfb = 0;
    if (captured) {
      cudaGraph_t g;
      const cudaGraphNode_t *deps = nullptr;
      size_t nd = 0;
      unsigned long long id;
      CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
      CK(cudaGraphConditionalHandleCreate(&cond2, g, 0, cudaGraphCondAssignDefault));
      if (check_nn) CK(cudaGraphConditionalHandleCreate(&condfb, g, 0, cudaGraphCondAssignDefault));
    }
    launch_pdl(pgm::k_cg_setup, grid1(nsys, 64), 64, 0, st, d_cg.p, nsys, mode == 0 ? (const int32_t *)ind->count : nullptr,
               (const double *)ind->norm, mode == 0 ? K : 0, set.fused, std::max(1, set.norm_refresh), mode, cond2, captured ? 1 : 0,
               use_nn ? 1 : 0);
    if (mode == 1) {
      // x0 = ind->mu with the plain start: X = mu, have = 1
      pgm::k_energy_start<T><<<grid1(nt), 256, 0, st>>>(a, ind->mu);
      check_launch();
    } else {
      last_hist = ind->hist;
      if (use_nn && !nn_forked) nn_fork(st, a, ind->hist);
      if (use_nn) {
        CK(cudaStreamWaitEvent(st, ev_nn_join, 0));  // the prediction, computed beside the row build
        nn_forked = false;
      }
      launch_pdl(pgm::k_start1<T>, grid1(nt), 256, 0, st, a, (const double *)ind->hist, K, cc[0], cc[1], cc[2], cc[3],
                 use_nn ? (const float *)nn_mu.p : nullptr);
    }
    sweep<true, false, 0, 0>(st, a, D.p, Bv.p);
    launch_pdl(pgm::k_start2<T>, ntblk, 256, 0, st, a);
    auto plain_start = [&](cudaStream_t s2) {
      sweep<false, false, 2, 1>(s2, a, X.p, AP.p);
      launch_pdl(pgm::k_start3<T>, grid1(nt), 256, 0, s2, a);
    };
    if (captured) conditional_node(st, cond2, cudaGraphCondTypeIf, plain_start);
    else plain_start(st);
    if (set.local_niter > 0) {
      pgm::k_cg_init<T, false, true><<<ntblk, 256, 0, st>>>(a); check_launch();
      local_precond<0, 0>(st, a, 0, 0);
    } else {
      pgm::k_cg_init<T><<<ntblk, 256, 0, st>>>(a); check_launch();
    }
    launch_pdl(pgm::k_cg_begin, 1, 256, 0, st, d_cg.p, nsys, set.dipole_tol, set.max_iter, dany.p,
               mode == 0 && set.predictor == 5 ? nn_fb_factor : 0.0, 0, condfb, captured && check_nn ? 1 : 0, dfb.p);
    if (check_nn) {
      auto fallback = [&](cudaStream_t s2) {
        launch_pdl(pgm::k_fb_prep<T>, grid1(nt), 256, 0, s2, a, (const float *)nn_mu.p);
        sweep<false, false, 3, 1>(s2, a, D.p, AP.p);  // A delta
        if (set.local_niter > 0) {
          launch_pdl(pgm::k_cg_init<T, true, true>, ntblk, 256, 0, s2, a, (const float *)nn_mu.p);
          local_precond<3, 0>(s2, a, 0, 0);
        } else {
          launch_pdl(pgm::k_cg_init<T, true>, ntblk, 256, 0, s2, a, (const float *)nn_mu.p);
        }
        launch_pdl(pgm::k_cg_begin, 1, 256, 0, s2, d_cg.p, nsys, set.dipole_tol, set.max_iter, dany.p, nn_fb_factor, 1,
                   condfb, 0, (int *)nullptr);
      };
      if (captured) {
        conditional_node(st, condfb, cudaGraphCondTypeIf, fallback);
      } else {
        int h = 0;
        CK(cudaMemcpyAsync(h_any, dfb.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        h = *h_any;
        if (h) fallback(st);
      }
    }
    if (captured) {
      // captured: the first U iterations as plain kernel nodes (their kernels skip systems that
      // have converged; U = the iterations of the last host-driven solve - 2), then a conditional
      // while node whose body is one CG iteration.  The last check before the node and the body's
      // last kernel set the condition to "some system still iterating" (max_iter on the device).
      cudaGraph_t g;
      const cudaGraphNode_t *deps = nullptr;
      size_t nd = 0;
      unsigned long long id;
      CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
      const int U = std::max(0, std::min(last_iters - 2, set.max_iter));
      cudaGraphConditionalHandle cond;
      CK(cudaGraphConditionalHandleCreate(&cond, g, U > 0 ? 0 : 1, cudaGraphCondAssignDefault));
      for (int k = 0; k < U; ++k) iteration(st, a, cond, k == U - 1 ? 1 : 0);
      unrolled = U;
      conditional_node(st, cond, cudaGraphCondTypeWhile, [&](cudaStream_t s2) {
        long long l0 = launches;
        iteration(s2, a, cond, 1);
        per_iter = launches - l0;
      });
    } else {
      int it = 0;
      for (; it < set.max_iter; ++it) {
        if (!any_active(st)) break;
        long long l0 = launches;
        iteration(st, a, 0, 0);
        per_iter = launches - l0;
      }
      last_iters = it;
    }
    launch_pdl(pgm::k_cg_finish<T>, grid1(nt), 256, 0, st, a, mu_out, mode == 0 ? ind->hist : nullptr, mode == 0 ? 1 : 0);
    launch_pdl(pgm::k_cg_state_out, grid1(nsys, 64), 64, 0, st, (const pgm::CGSys *)d_cg.p, nsys, ind->count, ind->norm, iters,
               resid, a.status, mode == 0 ? 1 : 0, set.dipole_tol);
  }

  // Energies, forces and virial at fixed mu (forcefield.py:2362-2430).
  void energy_pass(cudaStream_t st, pgm::Dev<T> &a, const double *mu, double *energy, double *virial, bool shadow = false) {
    launch_pdl(pgm::k_total_dipoles<T>, grid1(nt), 256, 0, st, a, mu);
    if (shadow) {
      // the reciprocal energy and potential of delta alone (zero outside extended steps), into
      // Phi2 and the second accumulators
      CK(cudaMemsetAsync(d_eacc2.p, 0, sizeof(pgm::EnergyAcc) * nsys, st));
      pgm::Dev<T> a2 = a;
      a2.Phi = Phi2.p;
      a2.eacc = d_eacc2.p;
      pme<false, false, 0, true>(st, a2, Dl.p);
    }
    pme<true, false, 0, true>(st, a, D.p);
    forces_pass(st, a, mu, true, 0, shadow);
    if (ncov) launch_pdl(pgm::k_cov_forces<T>, grid1(ncov), 256, 0, st, a);
    launch_pdl(pgm::k_energy_finish, grid1(nsys, 64), 64, 0, st, (const pgm::SysInfo *)d_sys.p, (const pgm::BoxInfo *)d_box.p,
               (const pgm::EnergyAcc *)d_eacc.p, nsys, set.ewald_beta, a.c_self, set.cutoff, set.vdw == 1, set.lj_lrc, a.induce, energy,
               virial, a.status, shadow ? (const pgm::EnergyAcc *)d_eacc2.p : (const pgm::EnergyAcc *)nullptr,
               set.iel_omega > 0 ? set.iel_omega : 1.0);
  }

  // The extended-Lagrangian step (forcefield.py:1558-1650) on the solver's kernels: per system a
  // warm-up solve to tol (plain start) or an extended step from x = xl[0] (fused start), then the
  // 0-SCF update or the CG iterations, the history push and the auxiliary dipoles' recurrence.
  void solve_iel(cudaStream_t st, pgm::Dev<T> &a, PgmInduction *ind, double *mu_out, int32_t *iters, double *resid) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cs));
    const bool captured = cs == cudaStreamCaptureStatusActive;
    cudaGraphConditionalHandle cond2 = 0, cond = 0;
    int U = 0;
    if (captured) {
      cudaGraph_t g;
      const cudaGraphNode_t *deps = nullptr;
      size_t nd = 0;
      unsigned long long id;
      CK(cudaStreamGetCaptureInfo(st, &cs, &id, &g, &deps, &nd));
      CK(cudaGraphConditionalHandleCreate(&cond2, g, 0, cudaGraphCondAssignDefault));
      U = std::max(0, std::min(last_iters - 2, set.max_iter));
      CK(cudaGraphConditionalHandleCreate(&cond, g, 0, cudaGraphCondAssignDefault));
    }
    launch_pdl(pgm::k_iel_setup, nsys, 256, 0, st, d_cg.p, (const pgm::SysInfo *)d_sys.p, nsys, (const int32_t *)ind->count,
               (const double *)ind->norm, (const double *)ind->mu, iel_warmup, set.iel, set.iel_iter, cond2, captured ? 1 : 0);
    launch_pdl(pgm::k_iel_start1<T>, grid1(nt), 256, 0, st, a, (const double *)ind->xl, (const double *)ind->mu);
    sweep<true, false, 0, 0>(st, a, D.p, Bv.p);
    launch_pdl(pgm::k_start2<T>, ntblk, 256, 0, st, a);
    auto plain_start = [&](cudaStream_t s2) {
      sweep<false, false, 2, 1>(s2, a, X.p, AP.p);
      launch_pdl(pgm::k_start3<T>, grid1(nt), 256, 0, s2, a);
    };
    if (captured) conditional_node(st, cond2, cudaGraphCondTypeIf, plain_start);
    else plain_start(st);
    pgm::k_cg_init<T><<<ntblk, 256, 0, st>>>(a); check_launch();
    launch_pdl(pgm::k_cg_begin, 1, 256, 0, st, d_cg.p, nsys, set.dipole_tol, set.max_iter, dany.p, 0.0, 0,
               (cudaGraphConditionalHandle)0, 0, (int *)nullptr);
    if (set.iel == 1) {
      const double om = set.iel_omega > 0 ? set.iel_omega : 1.0;
      launch_pdl(pgm::k_iel_delta<T>, grid1(nmol_total, 128), 128, 0, st, a, (const double *)ind->xl, om,
                 set.iel_precond == 0 ? 1 : 0, mu_out, Dl.p);
      launch_pdl(pgm::k_iel_begin, 1, 256, 0, st, d_cg.p, nsys, dany.p, 1, cond, (captured && U == 0) ? 1 : 0);
    } else if (captured && U == 0) {
      launch_pdl(pgm::k_iel_begin, 1, 256, 0, st, d_cg.p, nsys, dany.p, 0, cond, 1);  // the loop's condition only
    }
    if (captured) {
      for (int k = 0; k < U; ++k) iteration(st, a, cond, k == U - 1 ? 1 : 0);
      unrolled = U;
      conditional_node(st, cond, cudaGraphCondTypeWhile, [&](cudaStream_t s2) {
        long long l0 = launches;
        iteration(s2, a, cond, 1);
        per_iter = launches - l0;
      });
    } else {
      int it = 0;
      for (; it < set.max_iter; ++it) {
        if (!any_active(st)) break;
        long long l0 = launches;
        iteration(st, a, 0, 0);
        per_iter = launches - l0;
      }
      last_iters = it;
    }
    launch_pdl(pgm::k_iel_finish<T>, grid1(nt), 256, 0, st, a, mu_out, ind->hist, ind->xl, iel_co);
    launch_pdl(pgm::k_cg_state_out, grid1(nsys, 64), 64, 0, st, (const pgm::CGSys *)d_cg.p, nsys, ind->count, ind->norm, iters,
               resid, a.status, 1, set.dipole_tol);
  }

  void compute(cudaStream_t st, const double *pos, const double *box, const int32_t *idx, int idx_width, PgmInduction *ind,
               PgmOutputs *out) override {
    launches = 0;
    unsigned *status = out->status ? out->status : d_status.p;
    double *forces = out->forces ? out->forces : forces_tmp.p;
    pgm::Dev<T> a = dev(pos, idx, idx_width, forces, status);  // k_box zeroes the status words
    last_pos = pos;
    nn_forked = false;
    prepare(st, a, box, a.induce && set.predictor == 5 && nn_on ? ind->hist : nullptr);
    double *mu = ind->mu;
    if (a.induce && set.iel) {
      if (!ind->xl) throw CudaError{"iel: PgmInduction.xl (the auxiliary dipoles) is required"};
      solve_iel(st, a, ind, mu, out->iterations, out->residual);
    } else if (a.induce) {
      solve(st, a, ind, 0, mu, out->iterations, out->residual);
    } else {
      CK(cudaMemsetAsync(mu, 0, sizeof(double) * 3 * nt, st));
      if (out->iterations) CK(cudaMemsetAsync(out->iterations, 0, sizeof(int32_t) * nsys, st));
      if (out->residual) CK(cudaMemsetAsync(out->residual, 0, sizeof(double) * nsys, st));
    }
    energy_pass(st, a, mu, out->energy ? out->energy : energy_tmp.p, out->virial, a.induce && iel_shadow);
    if (!tune.tuned && !tune_fixed) {  // the first direct step: time the kernel variants on its rows
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      CK(cudaStreamIsCapturing(st, &cs));
      if (cs == cudaStreamCaptureStatusNone) autotune(st);
    }
  }

  void energy(cudaStream_t st, const double *pos, const double *box, const int32_t *idx, int idx_width, PgmInduction *ind,
              double *energy_out, int32_t *iters, uint32_t *status_out) override {
    launches = 0;
    unsigned *status = status_out ? status_out : d_status.p;
    CK(cudaMemsetAsync(status, 0, sizeof(unsigned) * nsys, st));
    pgm::Dev<T> a = dev(pos, idx, idx_width, forces_tmp.p, status);
    prepare(st, a, box);
    if (a.induce) {
      solve(st, a, ind, 1, ind->mu, iters, nullptr);
    } else {
      CK(cudaMemsetAsync(ind->mu, 0, sizeof(double) * 3 * nt, st));
      if (iters) CK(cudaMemsetAsync(iters, 0, sizeof(int32_t) * nsys, st));
    }
    energy_pass(st, a, ind->mu, energy_out, nullptr);
  }

  void fixed_mu(cudaStream_t st, const double *pos, const double *box, const int32_t *idx, int idx_width, const double *mu,
                double *energy_out, double *forces_out, double *virial, uint32_t *status_out) override {
    launches = 0;
    unsigned *status = status_out ? status_out : d_status.p;
    CK(cudaMemsetAsync(status, 0, sizeof(unsigned) * nsys, st));
    pgm::Dev<T> a = dev(pos, idx, idx_width, forces_out ? forces_out : forces_tmp.p, status);
    prepare(st, a, box);
    energy_pass(st, a, mu, energy_out ? energy_out : energy_tmp.p, virial);
  }

  void field(cudaStream_t st, const double *pos, const double *box, int with_q, const double *d, double *out) override {
    launches = 0;
    CK(cudaMemsetAsync(d_status.p, 0, sizeof(unsigned) * nsys, st));
    pgm::Dev<T> a = dev(pos, nullptr, 0, forces_tmp.p, d_status.p);
    prepare(st, a, box);
    pgm::k_load_vec<T><<<grid1(nt), 256, 0, st>>>(a, d, D.p); check_launch();
    if (with_q) sweep<true, false, 0, 0>(st, a, D.p, Bv.p);
    else sweep<false, false, 0, 0>(st, a, D.p, Bv.p);
    pgm::k_store_vec<T><<<grid1(nt), 256, 0, st>>>(a, Bv.p, out); check_launch();
  }
};

}  // namespace

struct PgmHandle {
  std::unique_ptr<EngineBase> eng;
  int device = 0;
  // pgm_compute_host: its own stream and, from the second call on, the force call replayed as a
  // captured graph (no host round trip per CG iteration) while the device buffers stay the same
  cudaStream_t host_stream = nullptr;
  cudaGraphExec_t host_graph = nullptr;
  long long host_graph_gen = -1;
  int host_calls = 0;
  ~PgmHandle() {
    if (host_graph) cudaGraphExecDestroy(host_graph);
    if (host_stream) cudaStreamDestroy(host_stream);
  }
};

static PgmStatus fail(PgmStatus s, const std::string &m) {
  g_err = m;
  return s;
}

extern "C" {

const char *pgm_last_error(void) { return g_err.c_str(); }

int pgm_iel_len(int order) {
  const int nc = order == 0 ? 1 : order + 1;
  return std::max(nc + 1, 3);
}

PgmStatus pgm_create(const PgmSettings *s, const PgmSystemDesc *systems, int n, int device, PgmHandle **out) {
  if (!s || !systems || n <= 0 || !out) return fail(PGM_ERR_INVALID, "null argument or no systems");
  if (s->iel < 0 || s->iel > 2) return fail(PGM_ERR_INVALID, "iel must be 0 (none), 1 (0scf) or 2 (scf)");
  if (s->iel && !(s->iel_order == 0 || (s->iel_order >= 3 && s->iel_order <= 9)))
    return fail(PGM_ERR_INVALID, "iel_order must be 0 or 3..9");
  if (s->iel && (s->iel_omega < 0 || s->iel_iter < 0 || s->iel_precond < 0 || s->iel_precond > 1))
    return fail(PGM_ERR_INVALID, "iel_omega >= 0, iel_iter >= 0, iel_precond 0 (block) or 1 (jacobi)");
  if (s->local_niter < 0 || s->local_niter > 8) return fail(PGM_ERR_INVALID, "local_niter must be 0..8");
  if (s->local_niter > 0 && s->iel)
    return fail(PGM_ERR_INVALID, "the local preconditioner (local_niter > 0) is not combined with iel");
  if (s->local_niter > 0 &&
      !(s->local_cut > 0 && s->local_cut < s->cutoff && (s->elec_cutoff <= 0 || s->local_cut < s->elec_cutoff)))
    return fail(PGM_ERR_INVALID, "local_cut must be positive and below the (electrostatics) cutoff");
  if (s->elec < 0 || s->elec > 3) return fail(PGM_ERR_INVALID, "elec must be 0..3 (q, qp, qi, qpi)");
  if (s->vdw < 0 || s->vdw > 1) return fail(PGM_ERR_INVALID, "vdw must be 0 (none) or 1 (lj)");
  if (s->precision < 0 || s->precision > 1) return fail(PGM_ERR_INVALID, "precision must be 0 (mixed) or 1 (double)");
  if (!(s->cutoff > 0) || !(s->ewald_beta > 0)) return fail(PGM_ERR_INVALID, "cutoff and ewald_beta must be positive");
  if (s->pme_order != 4 && s->pme_order != 6 && s->pme_order != 8) return fail(PGM_ERR_UNSUPPORTED, "pme_order must be 4, 6 or 8");
  if (s->predictor != 0 && s->predictor != 1 && s->predictor != 3 && s->predictor != 4 && s->predictor != 5)
    return fail(PGM_ERR_INVALID, "predictor must be 0 (none), 1 (previous step), 3 (mu3), 4 (mu4) or 5 (learned guess)");
  if (s->max_iter < 0) return fail(PGM_ERR_INVALID, "max_iter must be >= 0");
  if (s->elec_cutoff < 0 || s->elec_cutoff > s->cutoff)
    return fail(PGM_ERR_INVALID, "elec_cutoff must be 0 (none) or in (0, cutoff]");
  if (s->elec_capacity != 0 && !(s->elec_cutoff > 0 && s->elec_cutoff < s->cutoff && s->vdw))
    return fail(PGM_ERR_INVALID, "elec_capacity applies only to split rows (elec_cutoff < cutoff with a van der Waals term)");
  for (int i = 0; i < n; ++i) {
    const PgmSystemDesc &d = systems[i];
    if (d.n_atoms <= 0 || d.n_mol <= 0 || !d.mol_start || !d.q || !d.radius || !d.alpha || !d.lj_rmin_half || !d.lj_sqrt_eps ||
        !d.masses)
      return fail(PGM_ERR_INVALID, "system " + std::to_string(i) + ": missing arrays");
    if (d.mol_start[0] != 0 || d.mol_start[d.n_mol] != d.n_atoms) return fail(PGM_ERR_INVALID, "mol_start must span the atoms");
    for (int m = 0; m < d.n_mol; ++m)
      if (d.mol_start[m + 1] <= d.mol_start[m]) return fail(PGM_ERR_INVALID, "empty molecule");
    for (int a = 0; a < d.n_atoms; ++a)
      if (!(d.alpha[a] > 0)) return fail(PGM_ERR_UNSUPPORTED, "polarizabilities must be positive");
    for (int c = 0; c < d.n_cov; ++c)
      if (d.cov_i[c] < 0 || d.cov_i[c] >= d.n_atoms || d.cov_j[c] < 0 || d.cov_j[c] >= d.n_atoms)
        return fail(PGM_ERR_INVALID, "covalent dipole index out of range");
    for (int a = 0; a < 3; ++a) {
      int K = d.pme_grid[a];
      if (K < 2 * s->pme_order || K > 256 || K % 2 || radices(K).empty())
        return fail(PGM_ERR_UNSUPPORTED, "PME grid sizes must be even, 2, 3, 5-smooth, >= 2 order and <= 256");
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PGM_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(PGM_ERR_INVALID, "device index out of range");
  try {
    CK(cudaSetDevice(device));
    auto h = new PgmHandle();
    h->device = device;
    if (s->precision == 0) {
      if (s->pme_order == 4) h->eng.reset(new Engine<float, 4>());
      else if (s->pme_order == 6) h->eng.reset(new Engine<float, 6>());
      else h->eng.reset(new Engine<float, 8>());
    } else {
      if (s->pme_order == 4) h->eng.reset(new Engine<double, 4>());
      else if (s->pme_order == 6) h->eng.reset(new Engine<double, 6>());
      else h->eng.reset(new Engine<double, 8>());
    }
    if (s->precision == 0) {
      if (s->pme_order == 4) static_cast<Engine<float, 4> *>(h->eng.get())->init(s, systems, n);
      else if (s->pme_order == 6) static_cast<Engine<float, 6> *>(h->eng.get())->init(s, systems, n);
      else static_cast<Engine<float, 8> *>(h->eng.get())->init(s, systems, n);
    } else {
      if (s->pme_order == 4) static_cast<Engine<double, 4> *>(h->eng.get())->init(s, systems, n);
      else if (s->pme_order == 6) static_cast<Engine<double, 6> *>(h->eng.get())->init(s, systems, n);
      else static_cast<Engine<double, 8> *>(h->eng.get())->init(s, systems, n);
    }
    h->eng->nsys = n;
    *out = h;
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  } catch (std::exception &e) {
    return fail(PGM_ERR_CUDA, e.what());
  }
}

PgmStatus pgm_destroy(PgmHandle *h) {
  if (!h) return PGM_ERR_INVALID;
  cudaSetDevice(h->device);
  delete h;
  return PGM_OK;
}

PgmStatus pgm_compute(PgmHandle *h, void *stream, const double *pos, const double *box, const int32_t *idx, int idx_width,
                      PgmInduction *ind, PgmOutputs *out) {
  if (!h || !pos || !box || !ind || !out || !ind->mu) return fail(PGM_ERR_INVALID, "null argument");
  if (h->eng && (h->eng->nt > 0) && (!ind->hist || !ind->count || !ind->norm)) return fail(PGM_ERR_INVALID, "induction state incomplete");
  if (h->eng->iel_len && !ind->xl) return fail(PGM_ERR_INVALID, "iel: PgmInduction.xl (the auxiliary dipoles) is required");
  if (idx && idx_width <= 0) return fail(PGM_ERR_INVALID, "idx_width must be positive with idx");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->compute((cudaStream_t)stream, pos, box, idx, idx_width, ind, out);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_compute_host(PgmHandle *h, const double *pos, const double *box, PgmInduction *ind, PgmOutputs *out) {
  if (!h || !pos || !box || !out || (ind && (!ind->mu || !ind->hist || !ind->count || !ind->norm)))
    return fail(PGM_ERR_INVALID, "null argument");
  EngineBase *e = h->eng.get();
  if (ind && e->iel_len && !ind->xl) return fail(PGM_ERR_INVALID, "iel: PgmInduction.xl is required");
  size_t n3 = (size_t)3 * e->nt, ns = e->nsys, nxl = (size_t)e->iel_len * n3;
  double *d = nullptr;
  try {
    CK(cudaSetDevice(h->device));
    // one device block, kept by the handle: pos, box, mu, hist, norm, energy, forces, virial,
    // residual, (iEL) xl | count, iterations, status
    size_t nd = n3 + 9 * ns + n3 + 4 * n3 + ns + 3 * ns + n3 + 9 * ns + ns + nxl;
    size_t ni = 3 * ns;
    size_t bytes = sizeof(double) * nd + sizeof(int32_t) * ni;
    if (!h->host_stream) CK(cudaStreamCreateWithFlags(&h->host_stream, cudaStreamNonBlocking));
    if (e->host_scratch_bytes < bytes) {
      if (e->host_scratch) cudaFree(e->host_scratch);
      e->host_scratch = nullptr;
      e->host_scratch_bytes = 0;
      CK(cudaMalloc(&e->host_scratch, bytes));
      // a device-resident induction state starts empty (cleared on the stream of the calls)
      CK(cudaMemsetAsync(e->host_scratch, 0, bytes, h->host_stream));
      e->host_scratch_bytes = bytes;
      ++e->generation;
    }
    d = e->host_scratch;
    double *dpos = d, *dbox = dpos + n3, *dmu = dbox + 9 * ns, *dhist = dmu + n3, *dnorm = dhist + 4 * n3, *den = dnorm + ns,
           *dF = den + 3 * ns, *dvir = dF + n3, *dres = dvir + 9 * ns;
    double *dxl = dres + ns;
    int32_t *dcount = reinterpret_cast<int32_t *>(dxl + nxl), *dit = dcount + ns;
    uint32_t *dst = reinterpret_cast<uint32_t *>(dit + ns);
    cudaStream_t st = h->host_stream;
    CK(cudaMemcpyAsync(dpos, pos, sizeof(double) * n3, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(dbox, box, sizeof(double) * 9 * ns, cudaMemcpyHostToDevice, st));
    if (ind) {  // else the state the previous call left in the handle's block
      CK(cudaMemcpyAsync(dmu, ind->mu, sizeof(double) * n3, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(dhist, ind->hist, sizeof(double) * 4 * n3, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(dnorm, ind->norm, sizeof(double) * ns, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(dcount, ind->count, sizeof(int32_t) * ns, cudaMemcpyHostToDevice, st));
      if (nxl) CK(cudaMemcpyAsync(dxl, ind->xl, sizeof(double) * nxl, cudaMemcpyHostToDevice, st));
    }
    PgmInduction di{dmu, dhist, dcount, dnorm, nxl ? dxl : nullptr};
    PgmOutputs dout{den, dF, dvir, dit, dres, dst};
    if (h->host_graph && h->host_graph_gen != e->generation) {
      cudaGraphExecDestroy(h->host_graph);
      h->host_graph = nullptr;
    }
    if (!h->host_graph && h->host_calls > 0) {
      // capture once (the first call ran directly and sized the unrolled CG iterations)
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
      try {
        e->compute(st, dpos, dbox, nullptr, 0, &di, &dout);
      } catch (...) {
        cudaGraph_t junk;
        cudaStreamEndCapture(st, &junk);
        if (junk) cudaGraphDestroy(junk);
        throw;
      }
      cudaGraph_t g;
      CK(cudaStreamEndCapture(st, &g));
      cudaError_t ie = cudaGraphInstantiateWithFlags(&h->host_graph, g, cudaGraphInstantiateFlagUseNodePriority);
      cudaGraphDestroy(g);
      CK(ie);
      h->host_graph_gen = e->generation;
    }
    if (h->host_graph) CK(cudaGraphLaunch(h->host_graph, st));
    else e->compute(st, dpos, dbox, nullptr, 0, &di, &dout);
    ++h->host_calls;
    if (ind) {
      CK(cudaMemcpyAsync(ind->mu, dmu, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(ind->hist, dhist, sizeof(double) * 4 * n3, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(ind->norm, dnorm, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(ind->count, dcount, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, st));
      if (nxl) CK(cudaMemcpyAsync(ind->xl, dxl, sizeof(double) * nxl, cudaMemcpyDeviceToHost, st));
    }
    if (out->energy) CK(cudaMemcpyAsync(out->energy, den, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost, st));
    if (out->forces) CK(cudaMemcpyAsync(out->forces, dF, sizeof(double) * n3, cudaMemcpyDeviceToHost, st));
    if (out->virial) CK(cudaMemcpyAsync(out->virial, dvir, sizeof(double) * 9 * ns, cudaMemcpyDeviceToHost, st));
    if (out->iterations) CK(cudaMemcpyAsync(out->iterations, dit, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, st));
    if (out->residual) CK(cudaMemcpyAsync(out->residual, dres, sizeof(double) * ns, cudaMemcpyDeviceToHost, st));
    if (out->status) CK(cudaMemcpyAsync(out->status, dst, sizeof(uint32_t) * ns, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PGM_OK;
  } catch (CudaError &err) {
    return fail(PGM_ERR_CUDA, err.msg);
  }
}

PgmStatus pgm_energy(PgmHandle *h, void *stream, const double *pos, const double *box, const int32_t *idx, int idx_width,
                     PgmInduction *ind, double *energy, int32_t *iterations, uint32_t *status) {
  if (!h || !pos || !box || !ind || !ind->mu || !energy) return fail(PGM_ERR_INVALID, "null argument");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->energy((cudaStream_t)stream, pos, box, idx, idx_width, ind, energy, iterations, status);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_energy_fixed_mu(PgmHandle *h, void *stream, const double *pos, const double *box, const int32_t *idx,
                              int idx_width, const double *mu, double *energy, double *forces, double *virial,
                              uint32_t *status) {
  if (!h || !pos || !box || !mu) return fail(PGM_ERR_INVALID, "null argument");
  if (idx && idx_width <= 0) return fail(PGM_ERR_INVALID, "idx_width must be positive with idx");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->fixed_mu((cudaStream_t)stream, pos, box, idx, idx_width, mu, energy, forces, virial, status);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_field(PgmHandle *h, void *stream, const double *pos, const double *box, int with_charges, const double *d,
                    double *field) {
  if (!h || !pos || !box || !d || !field) return fail(PGM_ERR_INVALID, "null argument");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->field((cudaStream_t)stream, pos, box, with_charges, d, field);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_set_nn_model(PgmHandle *h, const float *weights, float sigma, float graph_cutoff) {
  if (!h || !(sigma > 0) || !(graph_cutoff > 0)) return fail(PGM_ERR_INVALID, "bad argument");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->set_nn(weights, sigma, graph_cutoff);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_tuning(PgmHandle *h, PgmTuning *out) {
  if (!h || !out) return fail(PGM_ERR_INVALID, "null argument");
  *out = h->eng->tuning();
  return PGM_OK;
}

PgmStatus pgm_set_tuning(PgmHandle *h, int rowfield_lanes, int forces_blocks_per_sm, int sweep_early, int rowfield_grid) {
  if (!h || !(rowfield_lanes == 0 || rowfield_lanes == 8 || rowfield_lanes == 16 || rowfield_lanes == 32) ||
      !(forces_blocks_per_sm == 0 || (forces_blocks_per_sm >= 2 && forces_blocks_per_sm <= 4)) || sweep_early < -1 ||
      sweep_early > 1 || rowfield_grid < -1 || rowfield_grid > 2)
    return fail(PGM_ERR_INVALID,
                "rowfield_lanes 0, 8, 16 or 32; forces_blocks_per_sm 0, 2, 3 or 4; sweep_early -1, 0 or 1; "
                "rowfield_grid -1, 0, 1 or 2");
  h->eng->set_tuning(rowfield_lanes, forces_blocks_per_sm, sweep_early, rowfield_grid);
  return PGM_OK;
}

PgmStatus pgm_autotune(PgmHandle *h, void *stream) {
  if (!h) return fail(PGM_ERR_INVALID, "null handle");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->autotune((cudaStream_t)stream);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_set_nn_fallback(PgmHandle *h, double factor) {
  if (!h || !(factor >= 0)) return fail(PGM_ERR_INVALID, "bad argument");
  h->eng->set_nn_fallback(factor);
  return PGM_OK;
}

PgmStatus pgm_nn_fallback_stats(PgmHandle *h, long long *fallbacks, double *ref_err) {
  if (!h) return fail(PGM_ERR_INVALID, "null handle");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->nn_fallback_stats(fallbacks, ref_err);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_set_mpnn_model(PgmHandle *h, const float *weights, float sigma, float graph_cutoff) {
  if (!h || !(sigma > 0) || !(graph_cutoff > 0)) return fail(PGM_ERR_INVALID, "bad argument");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->set_mpnn(weights, pgm_mpnn_param_count(), sigma, graph_cutoff);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_nn_graph(PgmHandle *h, void *stream, void *edges, int *counts, int emax) {
  if (!h || !edges || !counts || emax <= 0) return fail(PGM_ERR_INVALID, "bad argument");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->nn_graph((cudaStream_t)stream, (float4 *)edges, counts, emax);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_nn_features(PgmHandle *h, void *stream, const double *pos, const double *box, const double *hist,
                          const float *bl_prev, float *bl_out, float *inv, float *vec) {
  if (!h || !pos || !box || !hist || !bl_out || !inv || !vec) return fail(PGM_ERR_INVALID, "null argument");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->nn_features((cudaStream_t)stream, pos, box, hist, bl_prev, bl_out, inv, vec);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

PgmStatus pgm_set_row_capacity(PgmHandle *h, int capacity) {
  if (!h || capacity < 0) return fail(PGM_ERR_INVALID, "bad capacity");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->set_capacity(capacity);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

int pgm_row_capacity(const PgmHandle *h) { return h ? h->eng->capacity() : -1; }

PgmStatus pgm_set_list_capacity(PgmHandle *h, int capacity) {
  if (!h || capacity < 0) return fail(PGM_ERR_INVALID, "bad capacity");
  try {
    CK(cudaSetDevice(h->device));
    h->eng->set_list_capacity(capacity);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

int pgm_list_capacity(const PgmHandle *h) { return h ? h->eng->list_capacity() : -1; }

long long pgm_list_rebuilds(PgmHandle *h) {
  if (!h) return -1;
  try {
    return h->eng->list_rebuilds();
  } catch (CudaError &e) {
    g_err = e.msg;
    return -1;
  }
}

PgmStatus pgm_set_elec_capacity(PgmHandle *h, int capacity) {
  if (!h || capacity < 0) return fail(PGM_ERR_INVALID, "bad argument");
  try {
    CK(cudaSetDevice(h->device));
    if (!h->eng->set_elec_capacity(capacity)) return fail(PGM_ERR_INVALID, "elec_capacity applies only to split rows");
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}
int pgm_elec_capacity(const PgmHandle *h) { return h ? h->eng->elec_capacity() : -1; }
int pgm_max_vdw_count(PgmHandle *h) {
  if (!h) return -1;
  try {
    return h->eng->max_vdw_count();
  } catch (CudaError &e) {
    g_err = e.msg;
    return -1;
  }
}

int pgm_max_row_count(PgmHandle *h) {
  if (!h) return -1;
  try {
    return h->eng->max_count();
  } catch (CudaError &e) {
    g_err = e.msg;
    return -1;
  }
}

int pgm_num_atoms(const PgmHandle *h) { return h ? h->eng->nt : -1; }
int pgm_num_systems(const PgmHandle *h) { return h ? h->eng->nsys : -1; }
long long pgm_last_launch_count(const PgmHandle *h) { return h ? h->eng->launches : -1; }
long long pgm_launches_per_iteration(const PgmHandle *h) { return h ? h->eng->launches_per_iteration() : -1; }
int pgm_unrolled_iterations(const PgmHandle *h) { return h ? h->eng->unrolled : -1; }

PgmStatus pgm_profile_kernel(PgmHandle *h, void *stream, int which, int reps, double *ms_per_launch) {
  if (!h || !ms_per_launch || reps <= 0 || which < 0 || which > 12) return fail(PGM_ERR_INVALID, "bad argument");
  if (which == 10 && !h->eng->has_hist()) return fail(PGM_ERR_INVALID, "no solve with a history has run");
  if (!static_cast<bool>(h->eng)) return fail(PGM_ERR_INVALID, "no engine");
  try {
    CK(cudaSetDevice(h->device));
    *ms_per_launch = h->eng->profile((cudaStream_t)stream, which, reps);
    return PGM_OK;
  } catch (CudaError &e) {
    return fail(PGM_ERR_CUDA, e.msg);
  }
}

long long pgm_row_pairs(PgmHandle *h) {
  if (!h) return -1;
  try {
    return h->eng->row_pairs();
  } catch (CudaError &e) {
    g_err = e.msg;
    return -1;
  }
}

}  // extern "C"
