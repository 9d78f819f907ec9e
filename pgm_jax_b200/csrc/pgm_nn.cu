// pgm_nn.cu -- the learned initial guess of the induced-dipole solve: a small MLP on rotation
// invariants whose outputs mix per-atom vector channels (equivariant in the vectors), with BF16
// tensor-core (WMMA, FP32 accumulation) forward and backward kernels and an Adam step.  The
// reference has no counterpart (its solver starts from the mu4 / mu3 / ls predictors,
// pgm_jax/md/forcefield.py:1917-2008).
//
// Model: h1 = silu(x W1 + b1), h2 = silu(h1 W2 + b2), c = h2 W3 + b3 (x: NN_IN invariants, hidden
// NN_HID, c: NN_OUT coefficients, the first NN_CH used); mu = sum_c c_c v_c over the atom's vector
// channels.  Weights: an FP32 master array; each CTA converts them to BF16 in shared memory.  In
// training a CTA of 4 warps runs a tile of 64 samples through all layers (each warp 16 rows); in
// inference a CTA runs 16 samples, each warp a 16-column slice of every layer.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <mma.h>

#include <string>

#include "../../include/pgm_b200.h"
#include "pgm_nn.cuh"

using namespace nvcuda;

namespace pgmnn {

constexpr int TILE = 64;
constexpr int THREADS = 128;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

struct Smem {
  __nv_bfloat16 w1[NN_IN * NN_HID], w2[NN_HID * NN_HID], w3[NN_HID * NN_OUT];
  __nv_bfloat16 x[TILE * NN_IN], a1[TILE * NN_HID], a2[TILE * NN_HID];
  __nv_bfloat16 dzb[TILE * NN_HID], dz3[TILE * NN_OUT];
  float z1[TILE * NN_HID], z2[TILE * NN_HID], out[TILE * NN_OUT], dA[TILE * NN_HID];
  float wscr[THREADS / 32][256];
  float err[TILE][3];
  float b1[NN_HID], b2[NN_HID], b3[NN_OUT];
};

// C[16 x N] (ldc) = A[16 x K] (row-major, lda) B[K x N] (row-major, ldb).
template <int N, int K>
__device__ __forceinline__ void warp_gemm(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, float *C, int ldc) {
#pragma unroll
  for (int n = 0; n < N; n += 16) {
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.0f);
#pragma unroll
    for (int k = 0; k < K; k += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
      wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
      wmma::load_matrix_sync(fa, A + k, lda);
      wmma::load_matrix_sync(fb, B + k * ldb + n, ldb);
      wmma::mma_sync(acc, fa, fb, acc);
    }
    wmma::store_matrix_sync(C + n, acc, ldc, wmma::mem_row_major);
  }
}

// C[16 x N] = A[16 x K] B^T with B stored row-major as [N x K] (ldb = K).
template <int N, int K>
__device__ __forceinline__ void warp_gemm_bt(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, float *C, int ldc) {
#pragma unroll
  for (int n = 0; n < N; n += 16) {
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.0f);
#pragma unroll
    for (int k = 0; k < K; k += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
      wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::col_major> fb;
      wmma::load_matrix_sync(fa, A + k, lda);
      wmma::load_matrix_sync(fb, B + n * ldb + k, ldb);
      wmma::mma_sync(acc, fa, fb, acc);
    }
    wmma::store_matrix_sync(C + n, acc, ldc, wmma::mem_row_major);
  }
}

// dW (M x N, row-major in global, FP32) += A^T D over the tile's samples: A (TILE x M), D (TILE x N).
template <int M, int N>
__device__ void weight_grad(Smem &s, const __nv_bfloat16 *A, const __nv_bfloat16 *D, float *dW) {
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int tt = warp; tt < (M / 16) * (N / 16); tt += THREADS / 32) {
    int mt = tt / (N / 16), nt = tt % (N / 16);
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.0f);
#pragma unroll
    for (int k = 0; k < TILE; k += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::col_major> fa;  // A^T
      wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> fb;
      wmma::load_matrix_sync(fa, A + k * M + mt * 16, M);
      wmma::load_matrix_sync(fb, D + k * N + nt * 16, N);
      wmma::mma_sync(acc, fa, fb, acc);
    }
    float *mine = s.wscr[warp];
    wmma::store_matrix_sync(mine, acc, 16, wmma::mem_row_major);
    __syncwarp();
    for (int e = lane; e < 256; e += 32) atomicAdd(&dW[(mt * 16 + e / 16) * N + nt * 16 + (e % 16)], mine[e]);
    __syncwarp();
  }
}

// FP32 -> BF16 of n floats (n a multiple of 4 * THREADS; 16-byte aligned source), 16-byte loads,
// all of a thread's loads issued before the first conversion.
template <int N>
__device__ __forceinline__ void stage_bf16(const float *src, __nv_bfloat16 *dst) {
  static_assert(N % (4 * THREADS) == 0, "whole float4 rounds");
  const float4 *s4 = reinterpret_cast<const float4 *>(src);
  __nv_bfloat162 *d2 = reinterpret_cast<__nv_bfloat162 *>(dst);
  float4 v[N / (4 * THREADS)];
#pragma unroll
  for (int k = 0; k < N / (4 * THREADS); ++k) v[k] = s4[threadIdx.x + k * THREADS];
#pragma unroll
  for (int k = 0; k < N / (4 * THREADS); ++k) {
    int t = threadIdx.x + k * THREADS;
    d2[2 * t] = __floats2bfloat162_rn(v[k].x, v[k].y);
    d2[2 * t + 1] = __floats2bfloat162_rn(v[k].z, v[k].w);
  }
}

// The weights into shared memory (BF16 matrices, FP32 biases); blockDim.x == THREADS.
__device__ void stage_weights(const NNWeights &w, __nv_bfloat16 *w1, __nv_bfloat16 *w2, __nv_bfloat16 *w3, float *b1, float *b2,
                              float *b3) {
  stage_bf16<NN_IN * NN_HID>(w.w1, w1);
  stage_bf16<NN_HID * NN_HID>(w.w2, w2);
  stage_bf16<NN_HID * NN_OUT>(w.w3, w3);
  for (int t = threadIdx.x; t < NN_HID; t += blockDim.x) { b1[t] = w.b1[t]; b2[t] = w.b2[t]; }
  for (int t = threadIdx.x; t < NN_OUT; t += blockDim.x) b3[t] = w.b3[t];
}

__device__ void load_weights(Smem &s, const NNWeights &w) { stage_weights(w, s.w1, s.w2, s.w3, s.b1, s.b2, s.b3); }

__device__ void load_x(Smem &s, const float *inv, int n0, int n) {
  for (int t = threadIdx.x; t < TILE * NN_IN; t += blockDim.x) {
    int r = t / NN_IN, i = n0 + r;
    s.x[t] = __float2bfloat16(i < n ? inv[(size_t)i * NN_IN + (t - r * NN_IN)] : 0.f);
  }
}

// Forward of one tile (s.x loaded): z1, a1, z2, a2 and out = c.
__device__ void forward_tile(Smem &s) {
  const int r0 = (threadIdx.x >> 5) * 16;
  warp_gemm<NN_HID, NN_IN>(s.x + r0 * NN_IN, NN_IN, s.w1, NN_HID, s.z1 + r0 * NN_HID, NN_HID);
  __syncthreads();
  for (int t = threadIdx.x; t < TILE * NN_HID; t += blockDim.x) {
    float z = s.z1[t] + s.b1[t % NN_HID];
    s.z1[t] = z;
    s.a1[t] = __float2bfloat16(silu(z));
  }
  __syncthreads();
  warp_gemm<NN_HID, NN_HID>(s.a1 + r0 * NN_HID, NN_HID, s.w2, NN_HID, s.z2 + r0 * NN_HID, NN_HID);
  __syncthreads();
  for (int t = threadIdx.x; t < TILE * NN_HID; t += blockDim.x) {
    float z = s.z2[t] + s.b2[t % NN_HID];
    s.z2[t] = z;
    s.a2[t] = __float2bfloat16(silu(z));
  }
  __syncthreads();
  warp_gemm<NN_OUT, NN_HID>(s.a2 + r0 * NN_HID, NN_HID, s.w3, NN_OUT, s.out + r0 * NN_OUT, NN_OUT);
  __syncthreads();
  for (int t = threadIdx.x; t < TILE * NN_OUT; t += blockDim.x) s.out[t] += s.b3[t % NN_OUT];
  __syncthreads();
}

// Inference: a CTA of 4 warps runs 16 samples at a time through the layers with the output columns
// split across the warps (layers 1 and 2: 16 hidden columns per warp; layer 3: the 16 coefficient
// columns that the channel mix uses, its K = 64 split in four and the partial products summed in
// shared memory), so that a sample's chain of dependent tensor-core steps is a quarter of a whole
// layer stack.  The weights come as BF16 matrices in global memory (converted once, k_to_bf16):
// each warp loads its six B fragments straight from there (L2), with no staging and no barrier.
// Same rounding points as the training forward (BF16 operands, FP32 accumulation).
constexpr int FWD_ROWS = 16;
constexpr int FWD_WARPS = THREADS / 32;
static_assert(NN_HID == 16 * FWD_WARPS && NN_CH <= 16, "one 16-column slice of each layer per warp");
struct FwdSmem {
  __nv_bfloat16 x[FWD_ROWS * NN_IN], a1[FWD_ROWS * NN_HID], a2[FWD_ROWS * NN_HID];
  float z[FWD_ROWS * NN_HID];            // layer outputs before the activation
  float zp[FWD_WARPS][FWD_ROWS * 16];    // layer-3 partial products
};

using FragB = wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major>;

// C (16 x 16, ldc) = A[16 x 16 K] (lda) times the K / 16 B fragments fb.
template <int KS>
__device__ __forceinline__ void warp_slice(const __nv_bfloat16 *A, int lda, const FragB (&fb)[KS], float *C, int ldc) {
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
  wmma::fill_fragment(acc, 0.0f);
#pragma unroll
  for (int k = 0; k < KS; ++k) {
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> fa;
    wmma::load_matrix_sync(fa, A + 16 * k, lda);
    wmma::mma_sync(acc, fa, fb[k], acc);
  }
  wmma::store_matrix_sync(C, acc, ldc, wmma::mem_row_major);
}

// BF16 copies of the three weight matrices of the flat FP32 array, packed: W1 | W2 | W3.
constexpr int NN_WB = NN_WB_ELEMS;
__global__ void k_to_bf16(NNWeights w, __nv_bfloat16 *out) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= NN_WB) return;
  float v;
  if (t < NN_IN * NN_HID) v = w.w1[t];
  else if (t < NN_IN * NN_HID + NN_HID * NN_HID) v = w.w2[t - NN_IN * NN_HID];
  else v = w.w3[t - NN_IN * NN_HID - NN_HID * NN_HID];
  out[t] = __float2bfloat16(v);
}

__global__ void __launch_bounds__(THREADS) k_forward(NNWeights w, const __nv_bfloat16 *wb, const float *inv, const float *vec,
                                                     int n, float *mu) {
  __shared__ __align__(128) FwdSmem s;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, c0 = 16 * warp;
  const __nv_bfloat16 *W1 = wb, *W2 = W1 + NN_IN * NN_HID, *W3 = W2 + NN_HID * NN_HID;
  // this warp's B fragments: layer 1 columns c0.., layer 2 columns c0.. (four K steps), layer 3
  // rows c0.. of the first 16 columns
  FragB f1[1], f2[NN_HID / 16], f3[1];
  wmma::load_matrix_sync(f1[0], W1 + c0, NN_HID);
#pragma unroll
  for (int k = 0; k < NN_HID / 16; ++k) wmma::load_matrix_sync(f2[k], W2 + 16 * k * NN_HID + c0, NN_HID);
  wmma::load_matrix_sync(f3[0], W3 + c0 * NN_OUT, NN_OUT);
  const float b1 = w.b1[c0 + (lane & 15)], b2 = w.b2[c0 + (lane & 15)];
  for (int r0 = blockIdx.x * FWD_ROWS; r0 < n; r0 += gridDim.x * FWD_ROWS) {
    // the channel vectors of the mix (threads 0..47: row t / 3, component t % 3) in flight
    // through the layers
    float v[NN_CH];
    const int mr = threadIdx.x / 3, ma = threadIdx.x - 3 * mr, mi = r0 + mr;
    const bool mixer = threadIdx.x < FWD_ROWS * 3 && mi < n;
    if (mixer) {
      const float *vp = vec + (size_t)mi * NN_CH * 3 + ma;
#pragma unroll
      for (int c = 0; c < NN_CH; ++c) v[c] = vp[3 * c];
    }
    for (int t = threadIdx.x; t < FWD_ROWS * NN_IN; t += THREADS) {
      int i = r0 + t / NN_IN;
      s.x[t] = __float2bfloat16(i < n ? inv[(size_t)r0 * NN_IN + t] : 0.f);
    }
    __syncthreads();  // x
    warp_slice<1>(s.x, NN_IN, f1, s.z + c0, NN_HID);
    __syncwarp();
    for (int e = lane; e < FWD_ROWS * 16; e += 32) {  // column c0 + (e & 15) == c0 + (lane & 15)
      int r = e >> 4, c = c0 + (e & 15);
      s.a1[r * NN_HID + c] = __float2bfloat16(silu(s.z[r * NN_HID + c] + b1));
    }
    __syncthreads();  // a1 complete
    warp_slice<NN_HID / 16>(s.a1, NN_HID, f2, s.z + c0, NN_HID);
    __syncwarp();
    for (int e = lane; e < FWD_ROWS * 16; e += 32) {
      int r = e >> 4, c = c0 + (e & 15);
      s.a2[r * NN_HID + c] = __float2bfloat16(silu(s.z[r * NN_HID + c] + b2));
    }
    __syncthreads();  // a2 complete
    // layer 3, coefficient columns 0..15: this warp's 16 rows of K
    warp_slice<1>(s.a2 + c0, NN_HID, f3, s.zp[warp], 16);
    __syncthreads();
    if (mixer) {
      float acc = 0.f;
#pragma unroll
      for (int c = 0; c < NN_CH; ++c) {
        const int e = mr * 16 + c;
        const float coef = ((s.zp[0][e] + s.zp[1][e]) + (s.zp[2][e] + s.zp[3][e])) + w.b3[c];
        acc += coef * v[c];
      }
      mu[3 * (size_t)mi + ma] = acc;
    }
    __syncthreads();  // x, z and zp are rewritten by the next tile
  }
}

// Loss sum_i |mu_i - t_i|^2 * inv_scale and its gradient with respect to the weights (added to g).
__global__ void __launch_bounds__(THREADS) k_train(NNWeights w, NNWeights g, const float *inv, const float *vec, const float *target,
                                                   int n, float inv_scale, double *loss) {
  extern __shared__ __align__(128) unsigned char raw[];
  Smem &s = *reinterpret_cast<Smem *>(raw);
  __shared__ float red[THREADS / 32];
  load_weights(s, w);
  int n0 = blockIdx.x * TILE;
  load_x(s, inv, n0, n);
  __syncthreads();
  forward_tile(s);
  // e = mu - t per sample
  float lsum = 0.f;
  for (int t = threadIdx.x; t < TILE * 3; t += blockDim.x) {
    int r = t / 3, a = t - 3 * r, i = n0 + r;
    float e = 0.f;
    if (i < n) {
      const float *v = vec + (size_t)i * NN_CH * 3;
      float mu = 0.f;
#pragma unroll
      for (int c = 0; c < NN_CH; ++c) mu += s.out[r * NN_OUT + c] * v[3 * c + a];
      e = mu - target[3 * (size_t)i + a];
      lsum += inv_scale * e * e;
    }
    s.err[r][a] = e;
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float v = 0.f;
    for (int k = 0; k < THREADS / 32; ++k) v += red[k];
    atomicAdd(loss, (double)v);
  }
  // dL/dc_c = 2 inv_scale e . v_c (FP32 in out, BF16 in dz3)
  for (int t = threadIdx.x; t < TILE * NN_OUT; t += blockDim.x) {
    int r = t / NN_OUT, c = t - r * NN_OUT, i = n0 + r;
    float gc = 0.f;
    if (i < n && c < NN_CH) {
      const float *v = vec + (size_t)i * NN_CH * 3 + 3 * c;
      gc = 2.f * inv_scale * (s.err[r][0] * v[0] + s.err[r][1] * v[1] + s.err[r][2] * v[2]);
    }
    s.out[t] = gc;
    s.dz3[t] = __float2bfloat16(gc);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < NN_OUT; c += blockDim.x) {
    float b = 0.f;
    for (int r = 0; r < TILE; ++r) b += s.out[r * NN_OUT + c];
    atomicAdd(&g.b3[c], b);
  }
  weight_grad<NN_HID, NN_OUT>(s, s.a2, s.dz3, g.w3);
  const int r0 = (threadIdx.x >> 5) * 16;
  // dA2 = dZ3 W3^T, dZ2 = dA2 silu'(z2)
  warp_gemm_bt<NN_HID, NN_OUT>(s.dz3 + r0 * NN_OUT, NN_OUT, s.w3, NN_OUT, s.dA + r0 * NN_HID, NN_HID);
  __syncthreads();
  for (int t = threadIdx.x; t < TILE * NN_HID; t += blockDim.x) {
    float d = s.dA[t] * dsilu(s.z2[t]);
    s.dA[t] = d;
    s.dzb[t] = __float2bfloat16(d);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < NN_HID; c += blockDim.x) {
    float b = 0.f;
    for (int r = 0; r < TILE; ++r) b += s.dA[r * NN_HID + c];
    atomicAdd(&g.b2[c], b);
  }
  weight_grad<NN_HID, NN_HID>(s, s.a1, s.dzb, g.w2);
  __syncthreads();
  // dA1 = dZ2 W2^T (into z2, no longer needed), dZ1 = dA1 silu'(z1)
  warp_gemm_bt<NN_HID, NN_HID>(s.dzb + r0 * NN_HID, NN_HID, s.w2, NN_HID, s.z2 + r0 * NN_HID, NN_HID);
  __syncthreads();
  for (int t = threadIdx.x; t < TILE * NN_HID; t += blockDim.x) {
    float d = s.z2[t] * dsilu(s.z1[t]);
    s.dA[t] = d;
    s.dzb[t] = __float2bfloat16(d);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < NN_HID; c += blockDim.x) {
    float b = 0.f;
    for (int r = 0; r < TILE; ++r) b += s.dA[r * NN_HID + c];
    atomicAdd(&g.b1[c], b);
  }
  weight_grad<NN_IN, NN_HID>(s, s.x, s.dzb, g.w1);
}

__global__ void k_adam(float *w, float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float gg = g[t];
  float mm = b1 * m[t] + (1.f - b1) * gg;
  float vv = b2 * v[t] + (1.f - b2) * gg * gg;
  m[t] = mm;
  v[t] = vv;
  w[t] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  g[t] = 0.f;
}

size_t smem_bytes() { return sizeof(Smem); }

cudaError_t set_attrs() {
  static bool done = false;
  if (done) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(Smem));
  if (e == cudaSuccess) done = true;
  return e;
}

cudaError_t nn_weights_bf16(const float *flat, __nv_bfloat16 *wb, cudaStream_t st) {
  k_to_bf16<<<(NN_WB + 255) / 256, 256, 0, st>>>(nn_view(const_cast<float *>(flat)), wb);
  return cudaGetLastError();
}

cudaError_t nn_predict_launch(const float *flat, const __nv_bfloat16 *wb, const float *inv, const float *vec, int n, float *mu,
                              cudaStream_t st, int priority) {
  if (n <= 0) return cudaSuccess;
  const int tiles = (n + FWD_ROWS - 1) / FWD_ROWS;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tiles);  // one 16-sample tile per CTA
  cfg.blockDim = dim3(THREADS);
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributePriority;
  at[0].val.priority = priority;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_forward, nn_view(const_cast<float *>(flat)), wb, inv, vec, n, mu);
}

thread_local std::string g_nn_err;

}  // namespace pgmnn

extern "C" {

int pgm_nn_param_count(void) { return pgmnn::NN_NPARAM; }

PgmStatus pgm_nn_predict(void *stream, const float *weights, const float *inv, const float *vec, int n, float *mu) {
  if (!weights || !inv || !vec || !mu || n < 0) return PGM_ERR_INVALID;
  // the BF16 weight copy in stream-ordered memory, converted and released on the caller's stream
  cudaStream_t st = (cudaStream_t)stream;
  __nv_bfloat16 *wb = nullptr;
  cudaError_t e = cudaMallocAsync(&wb, sizeof(__nv_bfloat16) * pgmnn::NN_WB, st);
  if (e == cudaSuccess) e = pgmnn::nn_weights_bf16(weights, wb, st);
  if (e == cudaSuccess) e = pgmnn::nn_predict_launch(weights, wb, inv, vec, n, mu, st, 0);
  if (wb) {
    cudaError_t f = cudaFreeAsync(wb, st);
    if (e == cudaSuccess) e = f;
  }
  if (e != cudaSuccess) {
    pgmnn::g_nn_err = cudaGetErrorString(e);
    return PGM_ERR_CUDA;
  }
  return PGM_OK;
}

PgmStatus pgm_nn_loss_grad(void *stream, const float *weights, const float *inv, const float *vec, const float *target, int n,
                           float inv_scale, float *grad, double *loss) {
  if (!weights || !inv || !vec || !target || !grad || !loss || n <= 0) return PGM_ERR_INVALID;
  cudaError_t e = pgmnn::set_attrs();
  if (e == cudaSuccess) {
    pgmnn::k_train<<<(n + pgmnn::TILE - 1) / pgmnn::TILE, pgmnn::THREADS, pgmnn::smem_bytes(), (cudaStream_t)stream>>>(
        pgmnn::nn_view(const_cast<float *>(weights)), pgmnn::nn_view(grad), inv, vec, target, n, inv_scale, loss);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    pgmnn::g_nn_err = cudaGetErrorString(e);
    return PGM_ERR_CUDA;
  }
  return PGM_OK;
}

PgmStatus pgm_nn_adam(void *stream, float *weights, float *grad, float *m, float *v, float lr, float beta1, float beta2, float eps,
                      int step) {
  if (!weights || !grad || !m || !v || step < 1) return PGM_ERR_INVALID;
  int n = pgmnn::NN_NPARAM;
  float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  pgmnn::k_adam<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(weights, grad, m, v, n, lr, beta1, beta2, eps, c1, c2);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    pgmnn::g_nn_err = cudaGetErrorString(e);
    return PGM_ERR_CUDA;
  }
  return PGM_OK;
}

const char *pgm_nn_last_error(void) { return pgmnn::g_nn_err.c_str(); }

}  // extern "C"
