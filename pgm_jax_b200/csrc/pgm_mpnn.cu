// pgm_mpnn.cu -- the learned guess's message-passing network: its dense layers on tcgen05 tensor
// cores (pgm_tc.cuh) and the exported entry points.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "../../include/pgm_b200.h"
#include "pgm_tc.cuh"

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
  if (!A || !W || !C || !err || M < 0 || lda < K || ldc < N || lda % 8 || (act != 0 && act != 1)) {
    g_tc_err = "pgm_tc_gemm: bad argument";
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

}  // extern "C"
