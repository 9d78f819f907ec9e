// pgm_mpnn.cu -- the learned guess's message-passing network on the short-range graph.
//
// Per atom i, from the features of the channel and feature passes (pgm_kernels.cuh: 16 rotation
// invariants inv_i and 15 vector channels v_i,c), on the graph of the row entries closer than the
// graph cutoff rg (the list the row build writes: per atom up to emax edges (x, y, z, partner)):
//   h0 = SiLU(W0 inv + b0)                                       16 -> 64
//   two message-passing layers, each a continuous-filter convolution (SchNet, Schuett et al. 2017):
//     g = W_g h                                                  64 -> 16 message features
//     s_i[r, f] = sum_(i,j) phi_r(d_ij) g_j[f]                   sums over the graph's edges
//     a_i[f] = sum_r W_f[f, r] s_i[r, f]                         filter psi_f(d) = sum_r W_f[f, r] phi_r(d)
//     u = SiLU(W_a [h; a] + b_a)                                 80 -> 64
//     h <- h + W_b u + b_b                                       64 -> 64 (residual)
//   c = W_o h + b_o                                              64 -> 16 (15 used)
//   prediction sigma sum_c c_c v_i,c                             (e nm; rotates with the system)
// phi_r(d) = exp(-((d - r rg / 7) 7 / rg)^2) (cos(pi d / rg) + 1) / 2, r = 0..7.  An edge costs one
// 32-byte read of g_j (16 BF16 features) however many radial functions there are.
// The dense layers run on the tcgen05 tensor cores (pgm_tc.cuh: BF16 operands, FP32 accumulation,
// bias / SiLU / residual in the epilogue); the edge sums and the readout on the CUDA cores.
// Training: the same forward with the pre-activations and the sums s kept, then the backward pass:
// activation gradients through the transposed weights on the tensor cores (BF16 operands), the
// transposed convolution (the graph is symmetric: d_ij = d_ji), and the weight gradients as FP32
// sums over the atoms of the batch on the CUDA cores.  The NumPy restatement
// (oracle/nn_oracle.py mpnn_*) rounds to BF16 at the same points.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "../../include/pgm_b200.h"
#include "pgm_tc.cuh"

namespace pgmmp {

constexpr int IN = 16, HID = 64, R = 8, F = 16, ZW = HID + F, COEF = 16, CH = 15;
// flat FP32 parameters: W0 (64 x 16), b0, [Wg (16 x 64), Wf (16 x 8), Wa (64 x 80), ba, Wb (64 x 64), bb] x 2,
// Wo (16 x 64), bo
constexpr int L_SIZE = F * HID + F * R + HID * ZW + HID + HID * HID + HID;
constexpr int NPARAM = HID * IN + HID + 2 * L_SIZE + COEF * HID + COEF;
// BF16 copies: forward (out x in) of W0, Wg, Wa, Wb, Wo
constexpr int WB_FWD = HID * IN + 2 * (F * HID + HID * ZW + HID * HID) + COEF * HID;

struct View {
  const float *W0, *b0, *Wg[2], *Wf[2], *Wa[2], *ba[2], *Wb[2], *bb[2], *Wo, *bo;
};
__host__ __device__ inline View view(const float *p) {
  View v;
  v.W0 = p; v.b0 = p + HID * IN;
  const float *q = v.b0 + HID;
  for (int l = 0; l < 2; ++l) {
    v.Wg[l] = q; v.Wf[l] = q + F * HID; v.Wa[l] = v.Wf[l] + F * R; v.ba[l] = v.Wa[l] + HID * ZW;
    v.Wb[l] = v.ba[l] + HID; v.bb[l] = v.Wb[l] + HID * HID;
    q = v.bb[l] + HID;
  }
  v.Wo = q; v.bo = q + COEF * HID;
  return v;
}
// the gradient has the same layout
struct GView {
  float *W0, *b0, *Wg[2], *Wf[2], *Wa[2], *ba[2], *Wb[2], *bb[2], *Wo, *bo;
};
inline GView gview(float *p) {
  View v = view(p);
  GView g;
  g.W0 = const_cast<float *>(v.W0); g.b0 = const_cast<float *>(v.b0);
  for (int l = 0; l < 2; ++l) {
    g.Wg[l] = const_cast<float *>(v.Wg[l]); g.Wf[l] = const_cast<float *>(v.Wf[l]);
    g.Wa[l] = const_cast<float *>(v.Wa[l]); g.ba[l] = const_cast<float *>(v.ba[l]);
    g.Wb[l] = const_cast<float *>(v.Wb[l]); g.bb[l] = const_cast<float *>(v.bb[l]);
  }
  g.Wo = const_cast<float *>(v.Wo); g.bo = const_cast<float *>(v.bo);
  return g;
}

// BF16 weights: forward copies (out x in) and, for the backward pass, transposed copies (in x out);
// every matrix starts on a 16-byte boundary (its element count is a multiple of 8).
struct WB {
  __nv_bfloat16 *W0, *Wg[2], *Wa[2], *Wb[2], *Wo;        // forward
  __nv_bfloat16 *WgT[2], *WaT[2], *WbT[2], *WoT;          // transposed
};
constexpr int WB_ELEMS = WB_FWD + 2 * (HID * F + ZW * HID + HID * HID) + HID * COEF;
inline WB wb_view(__nv_bfloat16 *p) {
  WB w;
  w.W0 = p; p += HID * IN;
  for (int l = 0; l < 2; ++l) { w.Wg[l] = p; p += F * HID; w.Wa[l] = p; p += HID * ZW; w.Wb[l] = p; p += HID * HID; }
  w.Wo = p; p += COEF * HID;
  for (int l = 0; l < 2; ++l) { w.WgT[l] = p; p += HID * F; w.WaT[l] = p; p += ZW * HID; w.WbT[l] = p; p += HID * HID; }
  w.WoT = p;
  return w;
}

// (out x in) FP32 -> BF16 as is and transposed
__global__ void k_convert(const float *W, int out, int in, __nv_bfloat16 *Wf, __nv_bfloat16 *Wt) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= out * in) return;
  int o = t / in, i = t - o * in;
  __nv_bfloat16 b = __float2bfloat16(W[t]);
  if (Wf) Wf[t] = b;
  if (Wt) Wt[(size_t)i * out + o] = b;
}

// Radial functions of an edge of length d (float, as the NumPy restatement).
__device__ __forceinline__ float radial(int r, float d, float rg) {
  const float mu = r * (rg / (R - 1)), gam = ((R - 1) / rg) * ((R - 1) / rg);
  const float fc = 0.5f * (cospif(d / rg) + 1.0f);  // cos(pi d / rg), d / rg in [0, 1]
  const float x = d - mu;
  return expf(-gam * x * x) * fc;
}

// Eight floats rounded to BF16, packed for one 16-byte store.
__device__ __forceinline__ int4 pack_bf16x8(const float *x) {
  int4 o;
  int *w = &o.x;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const __nv_bfloat162 b = __floats2bfloat162_rn(x[2 * k], x[2 * k + 1]);
    w[k] = *reinterpret_cast<const int *>(&b);
  }
  return o;
}

// acc[f] += ph * (16 BF16 values of q0, q1)
__device__ __forceinline__ void fma_bf16x16(float *acc, float ph, int4 q0, int4 q1) {
  const __nv_bfloat162 *b0 = reinterpret_cast<const __nv_bfloat162 *>(&q0);
  const __nv_bfloat162 *b1 = reinterpret_cast<const __nv_bfloat162 *>(&q1);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float2 u = __bfloat1622float2(b0[k]), v = __bfloat1622float2(b1[k]);
    acc[2 * k] += ph * u.x;
    acc[2 * k + 1] += ph * u.y;
    acc[8 + 2 * k] += ph * v.x;
    acc[8 + 2 * k + 1] += ph * v.y;
  }
}

// The edge sums of one warp per atom.  Edges in blocks of 32: lane l loads edge b0 + l and evaluates
// its length and cosine cutoff once; then rounds of four edges: lane 8 s + r takes edge t + s
// (its length, cutoff and partner by shuffles) and radial r, and accumulates phi_r(d) x[partner][f]
// for the F = 16 values x of the partner (LOAD fetches them; the 8 lanes of an edge read the same
// 32 or 64 bytes).  After the loop each lane holds its slot's share of the sums over r.  A partner
// index outside [0, n) is skipped.
template <typename Load>
__device__ __forceinline__ void edge_sums(const float4 *__restrict__ e, int ne, int n, int self, float rg, int lane, float *acc,
                                          Load &&load) {
  const int s = lane >> 3, r = lane & 7;
  const float mu = r * (rg / (R - 1)), gam = ((R - 1) / rg) * ((R - 1) / rg);
  for (int b0 = 0; b0 < ne; b0 += 32) {
    float dl = 0.f, fcl = 0.f;
    int jl = self;
    if (b0 + lane < ne) {
      const float4 ed = __ldg(e + b0 + lane);
      const int j = __float_as_int(ed.w);
      if ((unsigned)j < (unsigned)n) {
        dl = sqrtf(ed.x * ed.x + ed.y * ed.y + ed.z * ed.z);
        fcl = 0.5f * (cospif(dl / rg) + 1.0f);
        jl = j;
      }
    }
    const int nb = min(32, ne - b0);
    for (int t = 0; t < nb; t += 4) {
      const float d = __shfl_sync(0xffffffffu, dl, t + s), fc = __shfl_sync(0xffffffffu, fcl, t + s);
      const int j = __shfl_sync(0xffffffffu, jl, t + s);
      const float x = d - mu;
      load(j, __expf(-gam * x * x) * fc, acc);  // lanes past the block's edges: fc = 0, j = self
    }
  }
#pragma unroll
  for (int o = 8; o < 32; o <<= 1)
#pragma unroll
    for (int f = 0; f < F; ++f) acc[f] += __shfl_xor_sync(0xffffffffu, acc[f], o);
}

// out[f] = sum_r W_f[f, r] acc_r[f] over the 8 lanes r of a slot (every lane ends with the sum).
__device__ __forceinline__ void filter_sum(float *acc, const float *__restrict__ Wf, int r) {
#pragma unroll
  for (int f = 0; f < F; ++f) acc[f] *= __ldg(Wf + f * R + r);
#pragma unroll
  for (int o = 1; o < 8; o <<= 1)
#pragma unroll
    for (int f = 0; f < F; ++f) acc[f] += __shfl_xor_sync(0xffffffffu, acc[f], o);
}

// The convolution of one layer, one warp per atom i: s_i[r, f] = sum over the atom's edges of
// phi_r(d) g_j[f] (G: n x 16 BF16, 16-byte aligned rows), a_i[f] = sum_r W_f[f, r] s_i[r, f] as
// BF16 into columns 64..79 of the atom's row of Z (ldz a multiple of 2); with S the sums s_i (n x 8
// x 16 FP32, for training).  Edges past emax are not read; a partner outside [0, n) is skipped.
//
// s_i = Phi^T G_i is a product over the edges (K), done with BF16 warp MMAs (m16n8k16, FP32
// accumulation): A = the radial values phi_r(d_e) rounded to BF16 (rows r = 0..7; rows 8..15
// zero), B = the partners' rows of G (16 edges x 16 features, two n8 tiles), read transposed from
// shared memory by ldmatrix.  The kernel is bound by the latency of its two dependent loads (edge
// list -> partner rows), so both go through asynchronous copies into shared memory (cp.async: many
// in flight per thread without registers): a warp walks atoms i, i + W, ... (W warps in the grid),
// copying the next atom's first 64 list slots while it works on the current one, and the partner
// rows of a 64-edge window (4 copies of 16 bytes per lane) are in flight while the radial values are
// formed.
constexpr int AGG_WARPS = 8, AGG_WIN = 64;
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
// slots s0 .. s0 + 63 of a list of emax slots (slots past emax: zeros; nothing past them is read)
__device__ __forceinline__ void agg_list(uint32_t dst, const float4 *__restrict__ e, int s0, int emax, int lane) {
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int sl = s0 + 32 * h + lane;
    cp_async16(dst + (uint32_t)(32 * h + lane) * 16u, sl < emax ? e + sl : e, sl < emax);
  }
}

__global__ void __launch_bounds__(32 * AGG_WARPS, 4) k_aggregate(const __nv_bfloat16 *__restrict__ G,
                                                              const float4 *__restrict__ edges,
                                                              const int *__restrict__ ecount, int emax, int n, float rg,
                                                              const float *__restrict__ Wf, __nv_bfloat16 *__restrict__ Z,
                                                              int ldz, float *__restrict__ S) {
  __shared__ __align__(16) __nv_bfloat16 tile[AGG_WARPS][AGG_WIN][F];  // partner rows of a window
  __shared__ __align__(16) float4 lists[AGG_WARPS][2][AGG_WIN];        // list slots, double-buffered
  __shared__ __align__(16) __nv_bfloat16 phis[AGG_WARPS][AGG_WIN][R];  // radial values of a window
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = gridDim.x * AGG_WARPS;
  int i = blockIdx.x * AGG_WARPS + wib;
  if (i >= n) return;  // whole warps leave: nothing below synchronises the block
  const int g = lane >> 2, tq = lane & 3;  // MMA fragment coordinates: row / column group
  const uint32_t tbase = (uint32_t)__cvta_generic_to_shared(&tile[wib][0][0]);
  const uint32_t lbase = (uint32_t)__cvta_generic_to_shared(&lists[wib][0][0]);
  const uint32_t pbase = (uint32_t)__cvta_generic_to_shared(&phis[wib][0][0]);
  int cur = 0;
  agg_list(lbase, edges + (size_t)i * emax, 0, emax, lane);
  cp_async_commit();
  int ne = min(ecount[i], emax);
  for (; i < n; i += nw) {
    const int inext = i + nw;
    if (inext < n) agg_list(lbase + (uint32_t)(1 - cur) * AGG_WIN * 16u, edges + (size_t)inext * emax, 0, emax, lane);
    cp_async_commit();  // (an empty group past the last atom keeps the count)
    const int nne = inext < n ? min(ecount[inext], emax) : 0;
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};  // n-tiles 0 (f 0..7) and 1 (f 8..15)
    for (int b0 = 0; b0 < ne; b0 += AGG_WIN) {
      if (b0 == 0) {
        cp_async_wait<1>();  // this atom's first slots (the next atom's may still be in flight)
      } else {               // windows past the first (long lists): copied and awaited here
        agg_list(lbase + (uint32_t)cur * AGG_WIN * 16u, edges + (size_t)i * emax, b0, emax, lane);
        cp_async_commit();
        cp_async_wait<0>();
      }
      __syncwarp();
      // per slot (lane, 32 + lane): partner and the 8 radial values as BF16 into the warp's phi tile
      // (phi_r = exp(-(t - r)^2) fc with t = 7 d / rg by the recurrence phi_r = phi_(r-1) q_r,
      // q_r = exp(2 t - 2 r + 1): two exponentials per edge; slots past the list: zeros, partner i)
      int jl[2];
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const float4 ed = lists[wib][cur][32 * w + lane];
        const int j = __float_as_int(ed.w);
        const bool ok = b0 + 32 * w + lane < ne && (unsigned)j < (unsigned)n;
        jl[w] = ok ? j : i;
        float ph[R];
#pragma unroll
        for (int r = 0; r < R; ++r) ph[r] = 0.f;
        if (ok) {
          const float r2 = ed.x * ed.x + ed.y * ed.y + ed.z * ed.z;
          const float d = r2 > 0.f ? r2 * rsqrtf(r2) : 0.f;
          const float fc = 0.5f * (__cosf(3.14159265f * d / rg) + 1.0f);
          const float t = d * ((R - 1) / rg);
          float v = __expf(-t * t) * fc, q = __expf(2.0f * t - 1.0f);
          ph[0] = v;
#pragma unroll
          for (int r = 1; r < R; ++r) {
            v *= q;
            q *= 0.135335283f;  // exp(-2)
            ph[r] = v;
          }
        }
        int4 pk;
        int *pw = &pk.x;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(ph[2 * k], ph[2 * k + 1]);
          pw[k] = *reinterpret_cast<const int *>(&b2);
        }
        *reinterpret_cast<int4 *>(&phis[wib][32 * w + lane][0]) = pk;
      }
      const int nq = min(4, (ne - b0 + 15) >> 4);  // 16-edge quarters of the window in use
      // partner rows: lane l copies half l & 1 of edge 16 q + (l >> 1) of quarter q
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q < nq) {
          const int j = __shfl_sync(0xffffffffu, jl[q >> 1], 16 * (q & 1) + (lane >> 1));
          cp_async16(tbase + (uint32_t)(((16 * q + (lane >> 1)) * F + 8 * (lane & 1)) * 2),
                     reinterpret_cast<const int4 *>(G + (size_t)j * F) + (lane & 1), true);
        }
      cp_async_commit();
      cp_async_wait<0>();  // the partner rows (and the next atom's slots, issued earlier)
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (q < nq) {
          const int m = lane >> 3, rr = lane & 7;
          // A: (edges 0-7, r 0-7) and (edges 8-15, r 0-7) of the phi tile, transposed: row g =
          // radial, columns 2 tq, 2 tq + 1 (+ 8) = edges
          uint32_t af[2];
          const uint32_t pa = pbase + (uint32_t)((16 * q + rr + 8 * (m & 1)) * R * 2);
          asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];"
                       : "=r"(af[0]), "=r"(af[1])
                       : "r"(pa));
          // B: (edges 0-7, f 0-7), (edges 8-15, f 0-7), (edges 0-7, f 8-15), (edges 8-15, f 8-15)
          const uint32_t addr = tbase + (uint32_t)(((16 * q + rr + 8 * (m & 1)) * F + 8 * (m >> 1)) * 2);
          uint32_t bq[4];
          asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];"
                       : "=r"(bq[0]), "=r"(bq[1]), "=r"(bq[2]), "=r"(bq[3])
                       : "r"(addr));
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
              "{%0, %1, %2, %3};"
              : "+f"(c0[0]), "+f"(c0[1]), "+f"(c0[2]), "+f"(c0[3])
              : "r"(af[0]), "r"(0u), "r"(af[1]), "r"(0u), "r"(bq[0]), "r"(bq[1]));
          asm volatile(
              "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
              "{%0, %1, %2, %3};"
              : "+f"(c1[0]), "+f"(c1[1]), "+f"(c1[2]), "+f"(c1[3])
              : "r"(af[0]), "r"(0u), "r"(af[1]), "r"(0u), "r"(bq[2]), "r"(bq[3]));
        }
      __syncwarp();  // the tile and the slots are rewritten by the next window or atom
    }
    if (ne == 0) cp_async_wait<1>();  // keep the group count in step for an atom without edges
    // lane (g, tq) holds s_i[g][2 tq + {0, 1}] (c0[0..1]) and s_i[g][8 + 2 tq + {0, 1}] (c1[0..1])
    if (S) {
      float *o = S + ((size_t)i * R + g) * F;
      *reinterpret_cast<float2 *>(o + 2 * tq) = make_float2(c0[0], c0[1]);
      *reinterpret_cast<float2 *>(o + 8 + 2 * tq) = make_float2(c1[0], c1[1]);
    }
    float v[4] = {c0[0] * __ldg(Wf + (2 * tq) * R + g), c0[1] * __ldg(Wf + (2 * tq + 1) * R + g),
                  c1[0] * __ldg(Wf + (8 + 2 * tq) * R + g), c1[1] * __ldg(Wf + (9 + 2 * tq) * R + g)};
#pragma unroll
    for (int o = 4; o < 32; o <<= 1)
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane < 4) {
      __nv_bfloat162 *z = reinterpret_cast<__nv_bfloat162 *>(Z + (size_t)i * ldz + HID);
      z[tq] = __floats2bfloat162_rn(v[0], v[1]);
      z[4 + tq] = __floats2bfloat162_rn(v[2], v[3]);
    }
    cur = 1 - cur;
    ne = nne;
  }
  cp_async_wait<0>();
}

// Grid of the edge-sum kernels: enough warps for every SM to hold its share at full occupancy,
// each warp walking atoms at the grid's stride.
inline int agg_blocks(int n) {
  static int resident = 0;  // blocks of k_aggregate that fit on the device at once
  if (!resident) {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_aggregate, 32 * AGG_WARPS, 0);
    resident = std::max(1, sms) * std::max(1, per);
  }
  return std::max(1, std::min((n + AGG_WARPS - 1) / AGG_WARPS, resident));
}

// The transposed convolution, one warp per atom j (the graph is symmetric): dg_j[f] = sum over j's
// edges (j, i) of psi_f(d) da_i[f], da = columns 64..79 of the rows of dZ (ldd a multiple of 4,
// 16-byte aligned), as FP32 (for the weight gradient) and BF16 (n x 16 each).
__global__ void __launch_bounds__(256) k_aggregate_t(const float *__restrict__ dZ, int ldd, const float4 *__restrict__ edges,
                                                     const int *__restrict__ ecount, int emax, int n, float rg,
                                                     const float *__restrict__ Wf, float *__restrict__ dG,
                                                     __nv_bfloat16 *__restrict__ dGb) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int j = warp;
  float acc[F];
#pragma unroll
  for (int f = 0; f < F; ++f) acc[f] = 0.f;
  edge_sums(edges + (size_t)j * emax, min(ecount[j], emax), n, j, rg, lane, acc, [&](int i, float ph, float *a) {
    const float4 *dp = reinterpret_cast<const float4 *>(dZ + (size_t)i * ldd + HID);
#pragma unroll
    for (int k = 0; k < F / 4; ++k) {
      const float4 v = __ldg(dp + k);
      a[4 * k] += ph * v.x; a[4 * k + 1] += ph * v.y; a[4 * k + 2] += ph * v.z; a[4 * k + 3] += ph * v.w;
    }
  });
  filter_sum(acc, Wf, lane & 7);
  if (lane == 0) {
    float4 *o = reinterpret_cast<float4 *>(dG + (size_t)j * F);
#pragma unroll
    for (int k = 0; k < F / 4; ++k) o[k] = make_float4(acc[4 * k], acc[4 * k + 1], acc[4 * k + 2], acc[4 * k + 3]);
    int4 *b = reinterpret_cast<int4 *>(dGb + (size_t)j * F);
    b[0] = pack_bf16x8(acc);
    b[1] = pack_bf16x8(acc + 8);
  }
}

// The filter weights' gradient: dWf[f, r] += sum_i da_i[f] s_i[r, f] (da: columns 64..79 of dZ);
// thread r F + f of a 128-thread block, atoms in a grid-stride loop, one atomic add per block.
__global__ void __launch_bounds__(R * F) k_wf_grad(const float *__restrict__ dZ, int ldd, const float *__restrict__ S, int n,
                                                   float *__restrict__ dWf) {
  const int t = threadIdx.x, r = t / F, f = t - r * F;
  float acc = 0.f;
  for (int i = blockIdx.x; i < n; i += gridDim.x) acc += dZ[(size_t)i * ldd + HID + f] * S[(size_t)i * R * F + t];
  atomicAdd(&dWf[f * R + r], acc);
}

// Prediction mu_i = sigma sum_c C[i, c] v[i, c] (FP32).
__global__ void k_readout(const float *__restrict__ C, const float *__restrict__ vec, int n, float sigma, float *__restrict__ mu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float m[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int c = 0; c < CH; ++c) {
    const float w = C[(size_t)i * COEF + c];
    for (int k = 0; k < 3; ++k) m[k] += w * vec[((size_t)i * CH + c) * 3 + k];
  }
  for (int k = 0; k < 3; ++k) mu[3 * (size_t)i + k] = sigma * m[k];
}

// Loss scale sum |mu - t|^2 (FP64 sum) and dC[i, c] = sigma (dL/dmu_i . v_ic) (0 for c = 15), as FP32
// and BF16.
__global__ void k_loss(const float *__restrict__ C, const float *__restrict__ vec, const float *__restrict__ target, int n,
                       float sigma, float scale, double *loss, float *__restrict__ dC, __nv_bfloat16 *__restrict__ dCb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < n) {
    float m[3] = {0.f, 0.f, 0.f};
    for (int c = 0; c < CH; ++c) {
      const float w = C[(size_t)i * COEF + c];
      for (int k = 0; k < 3; ++k) m[k] += w * vec[((size_t)i * CH + c) * 3 + k];
    }
    float dm[3];
    for (int k = 0; k < 3; ++k) {
      const float e = sigma * m[k] - target[3 * (size_t)i + k];
      l += (double)scale * e * e;
      dm[k] = 2.0f * scale * e;
    }
    for (int c = 0; c < COEF; ++c) {
      float v = 0.f;
      if (c < CH)
        for (int k = 0; k < 3; ++k) v += dm[k] * vec[((size_t)i * CH + c) * 3 + k];
      v *= sigma;
      dC[(size_t)i * COEF + c] = v;
      dCb[(size_t)i * COEF + c] = __float2bfloat16(v);
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
}

// u = BF16(SiLU(z)) into rows of ldu (training keeps z).
__global__ void k_silu_round(const float *__restrict__ z, int n, int w, __nv_bfloat16 *__restrict__ u, int ldu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * w) return;
  const int i = t / w, c = t - i * w;
  const float x = z[t];
  u[(size_t)i * ldu + c] = __float2bfloat16(__fdividef(x, 1.0f + __expf(-x)));
}

// dz = d * SiLU'(z) as FP32 and BF16.
__global__ void k_dsilu(const float *__restrict__ d, const float *__restrict__ z, int total, float *__restrict__ dz,
                        __nv_bfloat16 *__restrict__ dzb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= total) return;
  const float x = z[t], s = 1.0f / (1.0f + expf(-x));
  const float v = d[t] * s * (1.0f + x * (1.0f - s));
  dz[t] = v;
  if (dzb) dzb[t] = __float2bfloat16(v);
}

// dh (n x 64) += dZ[:, :64] (ld 80) + dGh (n x 64); also the BF16 copy of the new dh.
__global__ void k_add_dh(float *__restrict__ dh, const float *__restrict__ dZ, const float *__restrict__ dGh, int n,
                         __nv_bfloat16 *__restrict__ dhb) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * HID) return;
  const int i = t / HID, c = t - i * HID;
  const float v = dh[t] + dZ[(size_t)i * ZW + c] + dGh[t];
  dh[t] = v;
  dhb[t] = __float2bfloat16(v);
}

__global__ void k_to_bf16(const float *__restrict__ x, int total, __nv_bfloat16 *__restrict__ y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < total) y[t] = __float2bfloat16(x[t]);
}

// Weight gradients on the CUDA cores: dW[o, k] += sum_m dY[m, o] X[m, k] (X BF16, the first K of
// rows of ldx), db[o] += sum_m dY[m, o]; rows in chunks of 32 staged in shared memory, FP32 sums
// per thread, one atomic add per output and block.
template <int NO, int KI>
__global__ void __launch_bounds__(256) k_wgrad(const float *__restrict__ dY, int ldy, const __nv_bfloat16 *__restrict__ X, int ldx,
                                               int M, float *__restrict__ dW, float *__restrict__ db) {
  constexpr int CH_ROWS = 32;
  constexpr int PER = (NO * KI + 255) / 256;
  __shared__ float sY[CH_ROWS][NO];
  __shared__ float sX[CH_ROWS][KI];
  float acc[PER], accb = 0.f;
#pragma unroll
  for (int p = 0; p < PER; ++p) acc[p] = 0.f;
  for (int m0 = blockIdx.x * CH_ROWS; m0 < M; m0 += gridDim.x * CH_ROWS) {
    __syncthreads();
    for (int t = threadIdx.x; t < CH_ROWS * NO; t += 256) {
      const int r = t / NO, o = t - r * NO;
      sY[r][o] = m0 + r < M ? dY[(size_t)(m0 + r) * ldy + o] : 0.f;
    }
    for (int t = threadIdx.x; t < CH_ROWS * KI; t += 256) {
      const int r = t / KI, k = t - r * KI;
      sX[r][k] = m0 + r < M ? __bfloat162float(X[(size_t)(m0 + r) * ldx + k]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int e = threadIdx.x + 256 * p;
      if (e < NO * KI) {
        const int o = e / KI, k = e - o * KI;
        float s = 0.f;
#pragma unroll 8
        for (int r = 0; r < CH_ROWS; ++r) s += sY[r][o] * sX[r][k];
        acc[p] += s;
      }
    }
    if (db && threadIdx.x < NO)
      for (int r = 0; r < CH_ROWS; ++r) accb += sY[r][threadIdx.x];
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int e = threadIdx.x + 256 * p;
    if (e < NO * KI && acc[p] != 0.f) atomicAdd(&dW[e], acc[p]);
  }
  if (db && threadIdx.x < NO && accb != 0.f) atomicAdd(&db[threadIdx.x], accb);
}

// Workspace of the forward pass (inference) and of training, in bytes, for n atoms.
struct Work {
  __nv_bfloat16 *X0, *HZ[3], *Gb, *U;  // inputs; h with its message columns (n x 80) per layer; g (n x 16); u
  float *Cc;                           // coefficients (n x 16)
  // training only
  float *z0, *zu[2];                   // pre-activations
  __nv_bfloat16 *Gk[2], *Uk[2];        // g and u of both layers
  float *Sk[2];                        // the edge sums s (n x 8 x 16) of both layers
  float *dC, *dh, *dU, *dzu, *dZ, *dG, *dGh;
  __nv_bfloat16 *dCb, *dhb, *dzub, *dGb;
  __nv_bfloat16 *wb;                   // BF16 weights
  int *err;
};
inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
// The buffers in order (bytes); work_bytes and work_view walk the same list.
template <typename Take>
inline void work_layout(int n, bool train, Take &&take) {
  const size_t N = (size_t)n;
  take(N * IN * 2);
  for (int k = 0; k < 3; ++k) take(N * ZW * 2);
  take(N * F * 2); take(N * HID * 2);
  take(N * COEF * 4);
  if (train) {
    for (int k = 0; k < 3; ++k) take(N * HID * 4);       // z0, zu[0], zu[1]
    for (int k = 0; k < 2; ++k) take(N * F * 2);         // Gk
    for (int k = 0; k < 2; ++k) take(N * HID * 2);       // Uk
    for (int k = 0; k < 2; ++k) take(N * R * F * 4);     // Sk
    take(N * COEF * 4); take(N * HID * 4); take(N * HID * 4); take(N * HID * 4);  // dC, dh, dU, dzu
    take(N * ZW * 4); take(N * F * 4); take(N * HID * 4);                          // dZ, dG, dGh
    take(N * COEF * 2); take(N * HID * 2); take(N * HID * 2); take(N * F * 2);      // dCb, dhb, dzub, dGb
  }
  take((size_t)WB_ELEMS * 2);
  take(256);
}
inline size_t work_bytes(int n, bool train) {
  size_t b = 0;
  work_layout(n, train, [&](size_t bytes) { b += align256(bytes); });
  return b;
}
inline Work work_view(void *base, int n, bool train) {
  void *q[40];
  int k = 0;
  uint8_t *p = static_cast<uint8_t *>(base);
  work_layout(n, train, [&](size_t bytes) { q[k++] = p; p += align256(bytes); });
  Work w = {};
  int t = 0;
  auto bf = [&]() { return static_cast<__nv_bfloat16 *>(q[t++]); };
  auto fl = [&]() { return static_cast<float *>(q[t++]); };
  w.X0 = bf();
  for (int l = 0; l < 3; ++l) w.HZ[l] = bf();
  w.Gb = bf(); w.U = bf();
  w.Cc = fl();
  if (train) {
    w.z0 = fl(); w.zu[0] = fl(); w.zu[1] = fl();
    w.Gk[0] = bf(); w.Gk[1] = bf();
    w.Uk[0] = bf(); w.Uk[1] = bf();
    w.Sk[0] = fl(); w.Sk[1] = fl();
    w.dC = fl(); w.dh = fl(); w.dU = fl(); w.dzu = fl();
    w.dZ = fl(); w.dG = fl(); w.dGh = fl();
    w.dCb = bf(); w.dhb = bf(); w.dzub = bf(); w.dGb = bf();
  }
  w.wb = bf();
  w.err = static_cast<int *>(q[t++]);
  return w;
}

#define MPCK(x)                      \
  do {                               \
    cudaError_t e_ = (x);            \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

inline int blocks(long long n, int b = 256) { return (int)((n + b - 1) / b); }

cudaError_t convert_weights(const float *flat, Work &w, cudaStream_t st) {
  View v = view(flat);
  WB b = wb_view(w.wb);
  k_convert<<<blocks(HID * IN), 256, 0, st>>>(v.W0, HID, IN, b.W0, nullptr);
  for (int l = 0; l < 2; ++l) {
    k_convert<<<blocks(F * HID), 256, 0, st>>>(v.Wg[l], F, HID, b.Wg[l], b.WgT[l]);
    k_convert<<<blocks(HID * ZW), 256, 0, st>>>(v.Wa[l], HID, ZW, b.Wa[l], b.WaT[l]);
    k_convert<<<blocks(HID * HID), 256, 0, st>>>(v.Wb[l], HID, HID, b.Wb[l], b.WbT[l]);
  }
  k_convert<<<blocks(COEF * HID), 256, 0, st>>>(v.Wo, COEF, HID, b.Wo, b.WoT);
  return cudaGetLastError();
}

// The forward pass; with train, the pre-activations, every layer's g and u and the edge sums are kept.
cudaError_t forward(const float *flat, Work &w, const float *inv, const float4 *edges, const int *ecount, int emax, int n,
                    float rg, bool train, cudaStream_t st, int prio) {
  using namespace pgmtc;
  View v = view(flat);
  WB b = wb_view(w.wb);
  k_to_bf16<<<blocks((long long)n * IN), 256, 0, st>>>(inv, n * IN, w.X0);
  if (train) {
    MPCK((gemm<IN, HID, ACT_NONE, float>(w.X0, IN, n, b.W0, v.b0, w.z0, HID, w.err, st)));
    k_silu_round<<<blocks((long long)n * HID), 256, 0, st>>>(w.z0, n, HID, w.HZ[0], ZW);
  } else {
    MPCK((gemm<IN, HID, ACT_SILU, __nv_bfloat16>(w.X0, IN, n, b.W0, v.b0, w.HZ[0], ZW, w.err, st, nullptr, 0, prio)));
  }
  for (int l = 0; l < 2; ++l) {
    __nv_bfloat16 *H = w.HZ[l], *Hn = w.HZ[l + 1];
    __nv_bfloat16 *G = train ? w.Gk[l] : w.Gb, *U = train ? w.Uk[l] : w.U;
    MPCK((gemm<HID, F, ACT_NONE, __nv_bfloat16>(H, ZW, n, b.Wg[l], nullptr, G, F, w.err, st, nullptr, 0, prio)));
    k_aggregate<<<agg_blocks(n), 32 * AGG_WARPS, 0, st>>>(G, edges, ecount, emax, n, rg, v.Wf[l], H, ZW,
                                                                 train ? w.Sk[l] : nullptr);
    if (train) {
      MPCK((gemm<ZW, HID, ACT_NONE, float>(H, ZW, n, b.Wa[l], v.ba[l], w.zu[l], HID, w.err, st)));
      k_silu_round<<<blocks((long long)n * HID), 256, 0, st>>>(w.zu[l], n, HID, U, HID);
    } else {
      MPCK((gemm<ZW, HID, ACT_SILU, __nv_bfloat16>(H, ZW, n, b.Wa[l], v.ba[l], U, HID, w.err, st, nullptr, 0, prio)));
    }
    MPCK((gemm<HID, HID, ACT_NONE, __nv_bfloat16>(U, HID, n, b.Wb[l], v.bb[l], Hn, ZW, w.err, st, H, ZW, prio)));
  }
  MPCK((gemm<HID, COEF, ACT_NONE, float>(w.HZ[2], ZW, n, b.Wo, v.bo, w.Cc, COEF, w.err, st, nullptr, 0, prio)));
  return cudaGetLastError();
}

// ---- inference with the dense layers fused: three tile kernels (one CTA of 128 threads per 128
// atoms) around the two edge-sum launches.  IN: h0 = SiLU(W0 inv + b0) and g = W_g h0; MID (layer
// 0): u = SiLU(W_a [h0; a] + b_a), h1 = h0 + W_b u + b_b, g = W_g' h1; OUT (layer 1): u, h2 and
// c = W_o h2 + b_o with the readout mu = sigma sum_c c_c v_c.  The products of a tile run back to
// back on the tensor cores (u and h stay in shared memory, the accumulators in 64 TMEM columns),
// so only h (for the residual and the next layer), g and mu reach global memory.  The values are
// rounded to BF16 at the same points as the separate dense layers (forward()).
constexpr int FM_IN = 0, FM_MID = 1, FM_OUT = 2;
template <int MODE>
struct Fused {
  static constexpr int KA = MODE == FM_IN ? IN : ZW;    // K of the first product
  static constexpr int N3 = MODE == FM_OUT ? COEF : F;  // N of the last product
  static constexpr size_t A = (size_t)pgmtc::TM * KA * 2, W1 = (size_t)HID * KA * 2,
                          W2 = MODE == FM_IN ? 0 : (size_t)HID * HID * 2, UH = (size_t)pgmtc::TM * HID * 2,
                          W3 = (size_t)N3 * HID * 2;
  static constexpr size_t BIAS = (size_t)(HID + HID + COEF) * 4;  // b1, b2, b3 as FP32
  static constexpr size_t bytes = A + W1 + W2 + UH + W3 + BIAS + 64;
};
template <int K_, int N_>
struct KN {  // the shape of one product: K, N
  static constexpr int K = K_, N = N_;
};
struct FusedArgs {
  const float *inv;                  // IN: FP32 invariants (n x 16)
  const __nv_bfloat16 *Z;            // MID / OUT: h and a (n x 80)
  const __nv_bfloat16 *W1, *W2, *W3;  // W0 or W_a; W_b; W_g of the next layer or W_o (BF16, out x in)
  const float *b1, *b2, *b3;         // their biases (b3: null for W_g)
  __nv_bfloat16 *Hout;               // IN / MID: the new h into columns 0..63 of rows of ZW
  __nv_bfloat16 *Gout;               // IN / MID: g (n x 16)
  const float *vec;                  // OUT: channels (n x 15 x 3)
  float sigma;
  float *mu;                         // OUT: prediction (n x 3)
  int n;
  int *err;
};

template <int MODE>
__global__ void __launch_bounds__(pgmtc::THREADS) k_mp_fused(FusedArgs p) {
  using namespace pgmtc;
  using S = Fused<MODE>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sA = smem, *sW1 = sA + S::A, *sW2 = sW1 + S::W1, *sUH = sW2 + S::W2, *sW3 = sUH + S::UH;
  float *sb = reinterpret_cast<float *>(sW3 + S::W3);  // b1 (64), b2 (64), b3 (16)
  uint64_t *bar = reinterpret_cast<uint64_t *>(sW3 + S::W3 + S::BIAS);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  int *gave_up = reinterpret_cast<int *>(tslot + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * TM, row = m0 + tid, valid = min(TM, p.n - m0);
  const bool live = row < p.n;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(64));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    *gave_up = 0;
  }
  // weights (and the tile of Z) by asynchronous copies, all in flight together
  if constexpr (MODE != FM_IN) stage_async<TM, ZW>(sA, p.Z + (size_t)m0 * ZW, ZW, valid);
  stage_async<HID, S::KA>(sW1, p.W1, S::KA, HID);
  if constexpr (MODE != FM_IN) stage_async<HID, HID>(sW2, p.W2, HID, HID);
  stage_async<S::N3, HID>(sW3, p.W3, HID, S::N3);
  if constexpr (MODE == FM_IN) {  // FP32 invariants -> BF16: row tid, both halves loaded before either is stored
    float x[16];
    if (tid < valid) {
      const float4 *q = reinterpret_cast<const float4 *>(p.inv + (size_t)row * IN);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 u = q[k];
        x[4 * k] = u.x; x[4 * k + 1] = u.y; x[4 * k + 2] = u.z; x[4 * k + 3] = u.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) x[k] = 0.f;
    }
    st_bf16x8(sA + tile_off(tid, 0, IN), x);
    st_bf16x8(sA + tile_off(tid, 8, IN), x + 8);
  }
  for (int t = tid; t < HID + HID + COEF; t += THREADS) {
    float v = 0.f;  // absent biases (b2 of IN, b3 of W_g) as zeros
    if (t < HID) v = p.b1[t];
    else if (t < 2 * HID) { if (p.b2) v = p.b2[t - HID]; }
    else if (p.b3) v = p.b3[t - 2 * HID];
    sb[t] = v;
  }
  cp_async_wait_all();
  tc_barrier();
  const float *b1 = sb, *b2 = sb + HID, *b3 = sb + 2 * HID;
  const uint32_t tmem = *tslot, tl = tmem + ((uint32_t)(32 * warp) << 16), b = smem_u32(bar);
  uint32_t phase = 0;
  // a product into TMEM columns 0..N-1, then its wait (an abandoned wait stops the rest of the tile)
  auto product = [&](auto kn, uint32_t a0, uint32_t w0) -> bool {
    constexpr int K = decltype(kn)::K, N = decltype(kn)::N;
    if (*gave_up) return false;
    if (tid == 0) mma_issue<K, N>(tmem, a0, w0, b);
    __syncwarp();
    // one answer for the whole block: the epilogue's TMEM loads are warp-collective
    const bool ok = __syncthreads_and(mma_wait(b, phase, p.err));
    phase ^= 1u;
    if (!ok && tid == 0) *gave_up = 1;
    return ok;
  };
  using P1 = KN<S::KA, HID>;
  using P2 = KN<HID, HID>;
  using P3 = KN<HID, S::N3>;

  if (product(P1{}, smem_u32(sA), smem_u32(sW1))) {
#pragma unroll
    for (int c0 = 0; c0 < HID; c0 += 16) {
      float x[16];
      tmem_ld16(tl + c0, x);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float z = x[j] + b1[c0 + j];
        x[j] = __fdividef(z, 1.0f + __expf(-z));
      }
      // IN: h0 (global and the A operand of the last product); MID / OUT: u (A of the second)
      st_bf16x8(sUH + tile_off(tid, c0, HID), x);
      st_bf16x8(sUH + tile_off(tid, c0 + 8, HID), x + 8);
      if (MODE == FM_IN && live) {
        st_bf16x8(p.Hout + (size_t)row * ZW + c0, x);
        st_bf16x8(p.Hout + (size_t)row * ZW + c0 + 8, x + 8);
      }
    }
  }
  tc_barrier();
  if constexpr (MODE != FM_IN) {
    if (product(P2{}, smem_u32(sUH), smem_u32(sW2))) {
#pragma unroll
      for (int c0 = 0; c0 < HID; c0 += 16) {
        float x[16];
        tmem_ld16(tl + c0, x);
        const __nv_bfloat162 *hr0 = reinterpret_cast<const __nv_bfloat162 *>(sA + tile_off(tid, c0, ZW));
        const __nv_bfloat162 *hr1 = reinterpret_cast<const __nv_bfloat162 *>(sA + tile_off(tid, c0 + 8, ZW));
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const float2 u = __bfloat1622float2(hr0[k]), v = __bfloat1622float2(hr1[k]);
          x[2 * k] += b2[c0 + 2 * k] + u.x;
          x[2 * k + 1] += b2[c0 + 2 * k + 1] + u.y;
          x[8 + 2 * k] += b2[c0 + 8 + 2 * k] + v.x;
          x[8 + 2 * k + 1] += b2[c0 + 8 + 2 * k + 1] + v.y;
        }
        st_bf16x8(sUH + tile_off(tid, c0, HID), x);  // the second product is complete: u is free
        st_bf16x8(sUH + tile_off(tid, c0 + 8, HID), x + 8);
        if (MODE == FM_MID && live) {
          st_bf16x8(p.Hout + (size_t)row * ZW + c0, x);
          st_bf16x8(p.Hout + (size_t)row * ZW + c0 + 8, x + 8);
        }
      }
    }
    if constexpr (MODE == FM_OUT) {
      // the tile's channels (contiguous: 128 rows x 15 x 3 floats) into the free A and W1 regions,
      // in flight during the last product; read back per row without bank conflicts (stride 45)
      static_assert(S::A + S::W1 >= (size_t)TM * CH * 3 * 4, "room for the channels");
      __syncthreads();  // every thread is past its residual reads of the A region
      const int nbytes = valid * CH * 3 * 4;
      const char *src = reinterpret_cast<const char *>(p.vec + (size_t)m0 * CH * 3);
      for (int c = tid; c * 16 < nbytes; c += THREADS) {
        const int sz = min(16, nbytes - 16 * c);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(sA + 16 * c)), "l"(src + 16 * c),
                     "r"(sz)
                     : "memory");
      }
      asm volatile("cp.async.commit_group;" ::: "memory");
    }
    tc_barrier();
  }
  const bool ok3 = product(P3{}, smem_u32(sUH), smem_u32(sW3));
  if constexpr (MODE == FM_OUT) {  // the channels: own copies complete, then everyone's
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
  }
  if (ok3) {
    float x[16];
    tmem_ld16(tl, x);  // by every thread of the warp (a .sync.aligned load), live rows or not
    if (!live) {
    } else if constexpr (MODE == FM_OUT) {
      float m[3] = {0.f, 0.f, 0.f};
      const float *v = reinterpret_cast<const float *>(sA) + tid * CH * 3;
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        const float w = x[c] + b3[c];
#pragma unroll
        for (int k = 0; k < 3; ++k) m[k] += w * v[3 * c + k];
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) p.mu[3 * (size_t)row + k] = p.sigma * m[k];
    } else {
      st_bf16x8(p.Gout + (size_t)row * F, x);
      st_bf16x8(p.Gout + (size_t)row * F + 8, x + 8);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(64));
}

template <int MODE>
cudaError_t launch_fused(const FusedArgs &a, cudaStream_t st, int prio) {
  if (a.n <= 0) return cudaSuccess;
  const size_t sm = Fused<MODE>::bytes;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_mp_fused<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((a.n + pgmtc::TM - 1) / pgmtc::TM);
  cfg.blockDim = dim3(pgmtc::THREADS);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributePriority;
  at[0].val.priority = prio;
  cfg.attrs = at;
  cfg.numAttrs = prio ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_mp_fused<MODE>, a);
}

// Inference: mu (n x 3) from the invariants, channels and graph; five launches.
cudaError_t predict_fused(const float *flat, Work &w, const float *inv, const float *vec, const float4 *edges, const int *ecount,
                          int emax, int n, float sigma, float rg, float *mu, cudaStream_t st, int prio) {
  View v = view(flat);
  WB b = wb_view(w.wb);
  FusedArgs a = {};
  a.n = n;
  a.err = w.err;
  a.inv = inv;
  a.W1 = b.W0; a.b1 = v.b0; a.W3 = b.Wg[0];
  a.Hout = w.HZ[0]; a.Gout = w.Gb;
  MPCK(launch_fused<FM_IN>(a, st, prio));
  for (int l = 0; l < 2; ++l) {
    k_aggregate<<<agg_blocks(n), 32 * AGG_WARPS, 0, st>>>(w.Gb, edges, ecount, emax, n, rg, v.Wf[l], w.HZ[l], ZW,
                                                                 nullptr);
    FusedArgs m = {};
    m.n = n;
    m.err = w.err;
    m.Z = w.HZ[l];
    m.W1 = b.Wa[l]; m.b1 = v.ba[l]; m.W2 = b.Wb[l]; m.b2 = v.bb[l];
    if (l == 0) {
      m.W3 = b.Wg[1]; m.Hout = w.HZ[1]; m.Gout = w.Gb;
      MPCK(launch_fused<FM_MID>(m, st, prio));
    } else {
      m.W3 = b.Wo; m.b3 = v.bo; m.vec = vec; m.sigma = sigma; m.mu = mu;
      MPCK(launch_fused<FM_OUT>(m, st, prio));
    }
  }
  return cudaGetLastError();
}

// Loss and gradient (added into grad) of a batch whose forward pass ran with train.
cudaError_t backward(const float *flat, Work &w, const float *inv, const float *vec, const float *target, const float4 *edges,
                     const int *ecount, int emax, int n, float sigma, float rg, float scale, float *grad, double *loss,
                     cudaStream_t st) {
  using namespace pgmtc;
  (void)inv;
  View v = view(flat);
  GView g = gview(grad);
  WB b = wb_view(w.wb);
  const int wgb = std::min(blocks(n, 32), 1184);
  k_loss<<<blocks(n), 256, 0, st>>>(w.Cc, vec, target, n, sigma, scale, loss, w.dC, w.dCb);
  k_wgrad<COEF, HID><<<wgb, 256, 0, st>>>(w.dC, COEF, w.HZ[2], ZW, n, g.Wo, g.bo);
  MPCK((gemm<COEF, HID, ACT_NONE, float>(w.dCb, COEF, n, b.WoT, nullptr, w.dh, HID, w.err, st)));
  k_to_bf16<<<blocks((long long)n * HID), 256, 0, st>>>(w.dh, n * HID, w.dhb);
  for (int l = 1; l >= 0; --l) {
    // h_{l+1} = h_l + W_b u + b_b
    k_wgrad<HID, HID><<<wgb, 256, 0, st>>>(w.dh, HID, w.Uk[l], HID, n, g.Wb[l], g.bb[l]);
    MPCK((gemm<HID, HID, ACT_NONE, float>(w.dhb, HID, n, b.WbT[l], nullptr, w.dU, HID, w.err, st)));
    k_dsilu<<<blocks((long long)n * HID), 256, 0, st>>>(w.dU, w.zu[l], n * HID, w.dzu, w.dzub);
    k_wgrad<HID, ZW><<<wgb, 256, 0, st>>>(w.dzu, HID, w.HZ[l], ZW, n, g.Wa[l], g.ba[l]);
    MPCK((gemm<HID, ZW, ACT_NONE, float>(w.dzub, HID, n, b.WaT[l], nullptr, w.dZ, ZW, w.err, st)));
    k_wf_grad<<<std::min(n, 1184), R * F, 0, st>>>(w.dZ, ZW, w.Sk[l], n, g.Wf[l]);
    k_aggregate_t<<<blocks((long long)n * 32), 256, 0, st>>>(w.dZ, ZW, edges, ecount, emax, n, rg, v.Wf[l], w.dG, w.dGb);
    k_wgrad<F, HID><<<wgb, 256, 0, st>>>(w.dG, F, w.HZ[l], ZW, n, g.Wg[l], nullptr);
    MPCK((gemm<F, HID, ACT_NONE, float>(w.dGb, F, n, b.WgT[l], nullptr, w.dGh, HID, w.err, st)));
    k_add_dh<<<blocks((long long)n * HID), 256, 0, st>>>(w.dh, w.dZ, w.dGh, n, w.dhb);
  }
  k_dsilu<<<blocks((long long)n * HID), 256, 0, st>>>(w.dh, w.z0, n * HID, w.dzu, nullptr);
  k_wgrad<HID, IN><<<wgb, 256, 0, st>>>(w.dzu, HID, w.X0, IN, n, g.W0, g.b0);
  return cudaGetLastError();
}

__global__ void k_adam(float *w, float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.f - b1) * gt, vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  w[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
  g[t] = 0.f;
}

thread_local std::string g_mp_err;

}  // namespace pgmmp

namespace pgmmp_engine {
// For the engine (pgm_api.cu): predict mu on its stream from its features and graph.
size_t work_bytes(int n) { return pgmmp::work_bytes(n, false); }
cudaError_t set_weights(const float *flat, void *work, int n, cudaStream_t st) {
  pgmmp::Work w = pgmmp::work_view(work, n, false);
  (void)pgmmp::agg_blocks(n);  // the occupancy query once, before any stream capture
  cudaError_t e = cudaMemsetAsync(w.err, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  return pgmmp::convert_weights(flat, w, st);
}
cudaError_t predict(const float *flat, void *work, const float *inv, const float *vec, const float4 *edges, const int *ecount,
                    int emax, int n, float sigma, float rg, float *mu, cudaStream_t st, int prio) {
  pgmmp::Work w = pgmmp::work_view(work, n, false);
  return pgmmp::predict_fused(flat, w, inv, vec, edges, ecount, emax, n, sigma, rg, mu, st, prio);
}
}  // namespace pgmmp_engine

namespace {
thread_local std::string g_tc_err;

template <int K, int N>
cudaError_t tc_dispatch_act(int act, int out_f32, const __nv_bfloat16 *A, int lda, int M, const __nv_bfloat16 *W,
                            const float *bias, void *C, int ldc, int *err, cudaStream_t st) {
  if (out_f32) {
    if (act == pgmtc::ACT_SILU) return pgmtc::gemm<K, N, pgmtc::ACT_SILU, float>(A, lda, M, W, bias, (float *)C, ldc, err, st);
    return pgmtc::gemm<K, N, pgmtc::ACT_NONE, float>(A, lda, M, W, bias, (float *)C, ldc, err, st);
  }
  if (act == pgmtc::ACT_SILU)
    return pgmtc::gemm<K, N, pgmtc::ACT_SILU, __nv_bfloat16>(A, lda, M, W, bias, (__nv_bfloat16 *)C, ldc, err, st);
  return pgmtc::gemm<K, N, pgmtc::ACT_NONE, __nv_bfloat16>(A, lda, M, W, bias, (__nv_bfloat16 *)C, ldc, err, st);
}
}  // namespace

extern "C" {

const char *pgm_tc_last_error(void) { return g_tc_err.c_str(); }

PgmStatus pgm_tc_gemm(void *stream, int K, int N, int act, int out_f32, const void *A, int lda, int M, const void *W,
                      const float *bias, void *C, int ldc, int *err) {
  const bool misaligned = ((uintptr_t)A | (uintptr_t)W | (uintptr_t)C) % 16 != 0 || ldc % (out_f32 ? 4 : 8) != 0;
  if (!A || !W || !C || !err || M < 0 || lda < K || ldc < N || lda % 8 || misaligned || (act != 0 && act != 1)) {
    g_tc_err = "pgm_tc_gemm: bad argument (null pointer, negative size, or a stride or pointer off 16 bytes)";
    return PGM_ERR_INVALID;
  }
  const __nv_bfloat16 *a = (const __nv_bfloat16 *)A, *w = (const __nv_bfloat16 *)W;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (K == 16 && N == 64) e = tc_dispatch_act<16, 64>(act, out_f32, a, lda, M, w, bias, C, ldc, err, st);
  else if (K == 64 && N == 64) e = tc_dispatch_act<64, 64>(act, out_f32, a, lda, M, w, bias, C, ldc, err, st);
  else if (K == 64 && N == 128) e = tc_dispatch_act<64, 128>(act, out_f32, a, lda, M, w, bias, C, ldc, err, st);
  else if (K == 80 && N == 64) e = tc_dispatch_act<80, 64>(act, out_f32, a, lda, M, w, bias, C, ldc, err, st);
  else if (K == 64 && N == 32) e = tc_dispatch_act<64, 32>(act, out_f32, a, lda, M, w, bias, C, ldc, err, st);
  else if (K == 128 && N == 16) e = tc_dispatch_act<128, 16>(act, out_f32, a, lda, M, w, bias, C, ldc, err, st);
  else {
    g_tc_err = "pgm_tc_gemm: (K, N) not compiled";
    return PGM_ERR_UNSUPPORTED;
  }
  if (e != cudaSuccess) {
    g_tc_err = std::string("pgm_tc_gemm: ") + cudaGetErrorString(e);
    return PGM_ERR_CUDA;
  }
  return PGM_OK;
}

int pgm_mpnn_param_count(void) { return pgmmp::NPARAM; }
long long pgm_mpnn_work_bytes(int n, int train) { return (long long)pgmmp::work_bytes(n, train != 0); }
const char *pgm_mpnn_last_error(void) { return pgmmp::g_mp_err.c_str(); }

static PgmStatus mp_fail(PgmStatus s, const std::string &m) {
  pgmmp::g_mp_err = m;
  return s;
}

PgmStatus pgm_mpnn_predict(void *stream, const float *weights, const float *inv, const float *vec, const void *edges,
                           const int *ecount, int emax, int n, float sigma, float graph_cutoff, void *work, float *mu) {
  if (!weights || !inv || !vec || !edges || !ecount || !work || !mu || n <= 0 || emax <= 0 || !(graph_cutoff > 0))
    return mp_fail(PGM_ERR_INVALID, "pgm_mpnn_predict: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  pgmmp::Work w = pgmmp::work_view(work, n, false);
  cudaError_t e = cudaMemsetAsync(w.err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = pgmmp::convert_weights(weights, w, st);
  if (e == cudaSuccess)
    e = pgmmp::predict_fused(weights, w, inv, vec, (const float4 *)edges, ecount, emax, n, sigma, graph_cutoff, mu, st, 0);
  if (e != cudaSuccess) return mp_fail(PGM_ERR_CUDA, std::string("pgm_mpnn_predict: ") + cudaGetErrorString(e));
  return PGM_OK;
}

PgmStatus pgm_mpnn_loss_grad(void *stream, const float *weights, const float *inv, const float *vec, const float *target,
                             const void *edges, const int *ecount, int emax, int n, float sigma, float graph_cutoff,
                             float scale, void *work, float *grad, double *loss) {
  if (!weights || !inv || !vec || !target || !edges || !ecount || !work || !grad || !loss || n <= 0 || emax <= 0 ||
      !(graph_cutoff > 0))
    return mp_fail(PGM_ERR_INVALID, "pgm_mpnn_loss_grad: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  pgmmp::Work w = pgmmp::work_view(work, n, true);
  cudaError_t e = cudaMemsetAsync(w.err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = pgmmp::convert_weights(weights, w, st);
  if (e == cudaSuccess)
    e = pgmmp::forward(weights, w, inv, (const float4 *)edges, ecount, emax, n, graph_cutoff, true, st, 0);
  if (e == cudaSuccess)
    e = pgmmp::backward(weights, w, inv, vec, target, (const float4 *)edges, ecount, emax, n, sigma, graph_cutoff, scale, grad,
                        loss, st);
  if (e != cudaSuccess) return mp_fail(PGM_ERR_CUDA, std::string("pgm_mpnn_loss_grad: ") + cudaGetErrorString(e));
  return PGM_OK;
}

PgmStatus pgm_mpnn_adam(void *stream, float *weights, float *grad, float *m, float *v, float lr, float beta1, float beta2,
                        float eps, int step) {
  if (!weights || !grad || !m || !v || step < 1) return mp_fail(PGM_ERR_INVALID, "pgm_mpnn_adam: bad argument");
  const int n = pgmmp::NPARAM;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  pgmmp::k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(weights, grad, m, v, n, lr, beta1, beta2, eps, c1, c2);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mp_fail(PGM_ERR_CUDA, std::string("pgm_mpnn_adam: ") + cudaGetErrorString(e));
  return PGM_OK;
}

}  // extern "C"
