// pgm_nn.cuh -- sizes and weight layout of the learned initial guess (pgm_nn.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace pgmnn {

constexpr int NN_IN = 16;   // rotation invariants per atom
constexpr int NN_HID = 64;  // hidden width (2 layers)
constexpr int NN_OUT = 32;  // coefficient outputs (the first NN_CH used)
constexpr int NN_CH = 15;   // vector channels per atom
constexpr int NN_NPARAM = NN_IN * NN_HID + NN_HID + NN_HID * NN_HID + NN_HID + NN_HID * NN_OUT + NN_OUT;

// Views into one flat FP32 array, in this order: w1 (IN x HID), b1, w2 (HID x HID), b2,
// w3 (HID x OUT), b3 (row-major, x W convention).
struct NNWeights {
  float *w1, *b1, *w2, *b2, *w3, *b3;
};

inline __host__ __device__ NNWeights nn_view(float *flat) {
  NNWeights w;
  w.w1 = flat;
  w.b1 = w.w1 + NN_IN * NN_HID;
  w.w2 = w.b1 + NN_HID;
  w.b2 = w.w2 + NN_HID * NN_HID;
  w.w3 = w.b2 + NN_HID;
  w.b3 = w.w3 + NN_HID * NN_OUT;
  return w;
}

// BF16 copies of the weight matrices (W1 | W2 | W3, NN_WB elements) from the flat FP32 array.
constexpr int NN_WB_ELEMS = NN_IN * NN_HID + NN_HID * NN_HID + NN_HID * NN_OUT;
cudaError_t nn_weights_bf16(const float *flat, __nv_bfloat16 *wb, cudaStream_t st);

// mu (n, 3) FP32 = the model's prediction from invariants inv (n, NN_IN) and channels vec
// (n, NN_CH, 3), with the biases from the flat FP32 array and the matrices from their BF16 copy
// wb; launched on `st` (used by the engine's solver start).
cudaError_t nn_predict_launch(const float *flat, const __nv_bfloat16 *wb, const float *inv, const float *vec, int n, float *mu,
                              cudaStream_t st, int priority = 0);

}  // namespace pgmnn
