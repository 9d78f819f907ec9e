// pgm_tc.cuh -- dense layers of the learned guess on the 5th-generation tensor cores (sm_100a).
//
// C[M x N] = act(A[M x K] W[N x K]^T + bias): BF16 operands, FP32 accumulation in tensor memory.
// One CTA of 128 threads per 128-row tile of A: the tile and W are staged in shared memory in the
// K-major layout without swizzle (8-row x 16-byte core matrices, the two core matrices of one
// instruction's K = 16 adjacent: leading byte offset 128, stride byte offset (K / 8) x 128), one
// elected thread issues K / 16 tcgen05.mma (kind::f16, M = 128, N) into a TMEM accumulator of
// 128 lanes x N columns and commits them to an mbarrier; every warp then reads its 32 lanes with
// tcgen05.ld, adds the bias, applies the activation and stores its rows.
//
// Waits are bounded (a number of polls and 200 ms): a wait on the MMAs' mbarrier that gives up sets
// *err, waits once more (bounded) and still frees the tensor memory before returning.  The TMEM
// loads (warp-collective) are executed by every thread of a warp or by none.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgmtc {

constexpr int TM = 128;       // rows of A per tile (the MMA's M)
constexpr int THREADS = 128;  // four warps: warp w reads TMEM lanes 32 w .. 32 w + 31

// Activations of the epilogue.
constexpr int ACT_NONE = 0, ACT_SILU = 1;

// Shared-memory matrix descriptor of a K-major, unswizzled operand (sm_100 descriptor version 1):
// start address, leading byte offset (between the two core matrices adjacent in K), stride byte
// offset (between core matrices adjacent in M or N), all in 16-byte units.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// dense, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (r, k) of an R x K BF16 operand in that layout.
__host__ __device__ constexpr int tile_off(int r, int k, int K) {
  return (r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Tensor-memory columns for an N-column accumulator: a power of two, at least 32.
__host__ __device__ constexpr int tmem_cols(int N) { return N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256; }

// Shared memory of a tile: A (TM x K), W (N x K), the mbarrier and the TMEM address.
__host__ __device__ constexpr size_t smem_bytes(int K, int N) {
  return (size_t)TM * K * 2 + (size_t)N * K * 2 + 64;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Waits for phase `parity` of an mbarrier with at most `tries` polls and at most 200 ms; false when
// it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int tries) {
  const uint64_t t0 = global_ns();
  for (int t = 0; t < tries && global_ns() - t0 < 200000000ull; ++t) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

template <typename OutT>
__device__ __forceinline__ void store_val(OutT *p, float v);
template <>
__device__ __forceinline__ void store_val<float>(float *p, float v) { *p = v; }
template <>
__device__ __forceinline__ void store_val<__nv_bfloat16>(__nv_bfloat16 *p, float v) { *p = __float2bfloat16(v); }

// ---- building blocks of fused tile kernels (one CTA of THREADS threads per 128-row tile; thread t
// owns row t of the tile in every epilogue: warp w reads TMEM lanes 32 w .. 32 w + 31)

// Stages ROWS x K BF16 (rows of ld elements, 16-byte aligned; rows at or past `valid` as zeros)
// into the K-major core-matrix layout at dst.
template <int ROWS, int K>
__device__ __forceinline__ void stage_bf16(uint8_t *dst, const __nv_bfloat16 *__restrict__ src, int ld, int valid) {
  constexpr int KC = K / 8;
  for (int c = threadIdx.x; c < ROWS * KC; c += blockDim.x) {
    const int r = c / KC, kc = c - r * KC;
    int4 v = make_int4(0, 0, 0, 0);
    if (r < valid) v = *reinterpret_cast<const int4 *>(src + (size_t)r * ld + 8 * kc);
    *reinterpret_cast<int4 *>(dst + tile_off(r, 8 * kc, K)) = v;
  }
}

// The same with asynchronous copies (cp.async, 16 bytes each, zero-filled past `valid`): every
// copy of the thread in flight at once; cp_async_wait_all() before the tile is used.
template <int ROWS, int K>
__device__ __forceinline__ void stage_async(uint8_t *dst, const __nv_bfloat16 *__restrict__ src, int ld, int valid) {
  constexpr int KC = K / 8;
  for (int c = threadIdx.x; c < ROWS * KC; c += blockDim.x) {
    const int r = c / KC, kc = c - r * KC;
    const bool ok = r < valid;
    const __nv_bfloat16 *from = ok ? src + (size_t)r * ld + 8 * kc : src;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst + tile_off(r, 8 * kc, K))), "l"(from),
                 "r"(ok ? 16 : 0)
                 : "memory");
  }
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// K / 16 MMAs (M = 128, N, BF16, FP32 accumulation into TMEM columns tmem..tmem + N - 1) from
// K-major operands at shared addresses a0 (128 x K) and w0 (N x K); one thread issues them and
// commits to the mbarrier bar.
template <int K, int N>
__device__ __forceinline__ void mma_issue(uint32_t tmem, uint32_t a0, uint32_t w0, uint32_t bar) {
  const uint32_t id = idesc_bf16(TM, N);
#pragma unroll
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint64_t da = smem_desc(a0 + 256 * ks, 128, (K / 8) * 128);
    const uint64_t dw = smem_desc(w0 + 256 * ks, 128, (K / 8) * 128);
    const uint32_t acc = ks > 0 ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(da), "l"(dw), "r"(id), "r"(acc));
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 FP32 columns c0 .. c0 + 15 of this warp's 32 TMEM lanes (lane = row of the thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *x) {
  uint32_t v[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) x[j] = __uint_as_float(v[j]);
}

// Generic-proxy writes of shared memory made visible to the tensor core, and the block's threads
// (their tensor-memory reads included) ordered before what follows.
__device__ __forceinline__ void tc_barrier() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Waits for phase `parity` of the MMAs' mbarrier; on giving up sets *err, waits once more (also
// bounded) for the MMAs in flight, and returns false.
__device__ __forceinline__ bool mma_wait(uint32_t bar, uint32_t parity, int *err) {
  bool ok = mbar_wait(bar, parity, 1 << 22);
  if (!ok) {
    if ((threadIdx.x & 31) == 0) atomicExch(err, 1);
    mbar_wait(bar, parity, 1 << 22);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return ok;
}

// Eight floats rounded to BF16 and stored as one 16-byte access.
__device__ __forceinline__ void st_bf16x8(void *dst, const float *x) {
  int4 o;
  int *w = &o.x;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const __nv_bfloat162 b = __floats2bfloat162_rn(x[2 * k], x[2 * k + 1]);
    w[k] = *reinterpret_cast<const int *>(&b);
  }
  *reinterpret_cast<int4 *>(dst) = o;
}

// C = act(A W^T + bias) (+ Res) for one 128-row tile per CTA.  A: M rows of lda BF16 (the first K
// used), 16-byte aligned rows; W: N x K BF16 (K contiguous); bias: N floats or null; Res: null or
// M rows of ldr BF16 added after the activation (a residual connection); C: M rows of ldc.
// K: a multiple of 16 up to 256; N: a multiple of 16 up to 256; lda, ldr and ldc multiples of 8
// (each thread moves 16 values of its row with 16-byte accesses).
template <int K, int N, int ACT, typename OutT>
__global__ void __launch_bounds__(THREADS) k_tc_gemm(const __nv_bfloat16 *__restrict__ A, int lda, int M,
                                                     const __nv_bfloat16 *__restrict__ W, const float *__restrict__ bias,
                                                     OutT *__restrict__ C, int ldc, int *err,
                                                     const __nv_bfloat16 *__restrict__ Res = nullptr, int ldr = 0) {
  static_assert(K % 16 == 0 && K >= 16 && K <= 256, "K: a multiple of 16 up to 256");
  static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N: a multiple of 16 up to 256");
  constexpr int NCOL = tmem_cols(N);
  extern __shared__ __align__(1024) uint8_t smem[];
  uint8_t *sA = smem, *sW = smem + (size_t)TM * K * 2;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sW + (size_t)N * K * 2);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * TM;

  if (warp == 0) {  // the accumulator's columns (one warp allocates and frees)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  // stage the tile of A (rows past M as zeros) and W, 16 bytes (8 values of one core-matrix row) per
  // asynchronous copy
  stage_async<TM, K>(sA, A + (size_t)m0 * lda, lda, M - m0);
  stage_async<N, K>(sW, W, K, N);
  cp_async_wait_all();
  // the tensor core reads shared memory through the async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;

  if (tid == 0) {
    const uint32_t a0 = smem_u32(sA), w0 = smem_u32(sW), id = idesc_bf16(TM, N);
#pragma unroll
    for (int ks = 0; ks < K / 16; ++ks) {
      const uint64_t da = smem_desc(a0 + 256 * ks, 128, (K / 8) * 128);
      const uint64_t dw = smem_desc(w0 + 256 * ks, 128, (K / 8) * 128);
      const uint32_t acc = ks > 0 ? 1u : 0u;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "setp.ne.b32 p, %4, 0;\n\t"
          "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
          "l"(da), "l"(dw), "r"(id), "r"(acc));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
  }
  __syncwarp();
  bool ok = mbar_wait(smem_u32(bar), 0, 1 << 22);
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
    mbar_wait(smem_u32(bar), 0, 1 << 22);  // the MMAs in flight, once more, before the memory is freed
  }
  ok = __syncthreads_and(ok);  // one answer for the block: the TMEM loads below are warp-collective
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (ok) {
    const int row = m0 + 32 * warp + lane;
    const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
          "[%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
            "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        float x[16];
        __nv_bfloat16 rb[16];
        if (Res) {  // 2 x 16-byte loads of the residual row segment
          *reinterpret_cast<int4 *>(rb) = *reinterpret_cast<const int4 *>(Res + (size_t)row * ldr + c0);
          *reinterpret_cast<int4 *>(rb + 8) = *reinterpret_cast<const int4 *>(Res + (size_t)row * ldr + c0 + 8);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          x[j] = __uint_as_float(v[j]) + (bias ? bias[c0 + j] : 0.0f);
          if (ACT == ACT_SILU) x[j] = __fdividef(x[j], 1.0f + __expf(-x[j]));
          if (Res) x[j] += __bfloat162float(rb[j]);
        }
        OutT *dst = C + (size_t)row * ldc + c0;  // 16-byte aligned: ldc a multiple of 8, c0 of 16
        if constexpr (sizeof(OutT) == 2) {
          __nv_bfloat16 o[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) o[j] = __float2bfloat16(x[j]);
          reinterpret_cast<int4 *>(dst)[0] = *reinterpret_cast<const int4 *>(o);
          reinterpret_cast<int4 *>(dst)[1] = *reinterpret_cast<const int4 *>(o + 8);
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            reinterpret_cast<float4 *>(dst)[j] = make_float4(x[4 * j], x[4 * j + 1], x[4 * j + 2], x[4 * j + 3]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL));
}

// Launch: ceil(M / 128) CTAs of 128 threads with the tile's shared memory.
template <int K, int N, int ACT, typename OutT>
cudaError_t gemm(const __nv_bfloat16 *A, int lda, int M, const __nv_bfloat16 *W, const float *bias, OutT *C, int ldc, int *err,
                 cudaStream_t st, const __nv_bfloat16 *Res = nullptr, int ldr = 0, int priority = 0) {
  if (M <= 0) return cudaSuccess;
  const size_t sm = smem_bytes(K, N);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_tc_gemm<K, N, ACT, OutT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((M + TM - 1) / TM);
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributePriority;
  at[0].val.priority = priority;
  cfg.attrs = at;
  cfg.numAttrs = priority ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k_tc_gemm<K, N, ACT, OutT>, A, lda, M, W, bias, C, ldc, err, Res, ldr);
}

}  // namespace pgmtc
