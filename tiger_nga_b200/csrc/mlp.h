// The surrogate MLP's device state (shared by the training and inference translation units).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tng_runtime.h"

namespace tng {

constexpr int kMlpMaxHidden = 8;  // hidden layers at most

struct Mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  int n_in = 0, n_out = 0, in_pad = 0, out_pad = 0, hidden = 0, nlin = 0;
  int fan_in[kMlpMaxHidden + 1] = {}, fan_out[kMlpMaxHidden + 1] = {};
  int64_t w_off[kMlpMaxHidden + 1] = {}, b_off[kMlpMaxHidden + 1] = {};
  int64_t nparam = 0;
  float* params = nullptr;  // [W0 b0 W1 b1 ...], W_l row-major (fan_out x fan_in)
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  int64_t step = 0;
  // loss weight of outputs predicted below their target (1: plain weighted MSE); the error gate
  // is trained with a larger one, so that it errs on the side of over-predicting errors
  float under_weight = 1.f;
  DevBuf act, pre, work, part, lossp, gather;
};

int mlp_init(Mlp* m, int device, cudaStream_t stream, int n_in, int n_out, int hidden, int layers, uint64_t seed);
void mlp_free(Mlp* m);
int mlp_forward_f32(Mlp* m, const float* X, int rows, float** Y);
int mlp_backward(Mlp* m, const float* X, const float* T, const float* w_out, int rows, float* loss);
int mlp_adam(Mlp* m, float lr);
// Minibatch Adam with a cosine learning rate over `epochs` passes. An epoch visits the row
// indices of `pop` (host, npop entries, repeats allowed: a resampled population) in a fresh
// random order, or every row 0..n-1 when pop is null.
int mlp_train(Mlp* m, const float* X, const float* T, const float* w_out, int64_t n, int epochs, int batch, float lr0,
              uint64_t seed, float* losses, const int* pop = nullptr, int64_t npop = 0);

}  // namespace tng
