// The learned part of the PCG warm start: a small MLP (8 inputs, three tanh layers
// of 64, one linear output) with BF16 weights, trained on the GPU by this library's
// own fused forward/backward kernel and an Adam kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "engine.cuh"

namespace saige {

constexpr int kMlpIn = 8;
constexpr int kMlpH = 64;
// Parameter layout (FP32 master and BF16 copy alike):
//   W1 [H][IN], b1 [H], W2 [H][H], b2 [H], W3 [H][H], b3 [H], w4 [H], b4 [1]
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpH * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpH;
constexpr int kMlpB2 = kMlpW2 + kMlpH * kMlpH;
constexpr int kMlpW3 = kMlpB2 + kMlpH;
constexpr int kMlpB3 = kMlpW3 + kMlpH * kMlpH;
constexpr int kMlpW4 = kMlpB3 + kMlpH;
constexpr int kMlpB4 = kMlpW4 + kMlpH;
constexpr int kMlpParams = kMlpB4 + 1;

struct Mlp {
  DevBuf mem;
  DevBuf part, lpart;         // per-block gradient partials of the training pass
  int part_blocks = 0;
  cudaGraphExec_t graph = nullptr;  // captured training steps (see mlp_train)
  const void* graph_key[2] = {nullptr, nullptr};
  int64_t graph_n = 0;
  int graph_q = 0, graph_batch = 0, graph_holdout = 0, graph_steps = 0;
  float graph_lr = 0.f;
  ~Mlp() {
    if (graph) cudaGraphExecDestroy(graph);
  }
  float* master = nullptr;    // FP32 weights
  uint16_t* wbf = nullptr;    // BF16 copy used by the forward passes
  float* grad = nullptr;      // gradient accumulator
  float* m1 = nullptr;        // Adam moments
  float* m2 = nullptr;
  int* step = nullptr;        // device step counter (mini-batch offset, Adam bias correction)
  double* loss = nullptr;     // [2]: summed squared error of the last pass, example count
  bool ready = false;         // initialised
  int64_t trained_steps = 0;
};

// Allocates and initialises the weights (uniform +-1/sqrt(fan_in), from seed).
Status mlp_init(Mlp& m, uint64_t seed, cudaStream_t st);

// out[e] = MLP(F[e*8 .. e*8+8]) for e < n_ex (BF16 weights, FP32 arithmetic).
Status mlp_forward(const Mlp& m, const float* F, int64_t n_ex, float* out, cudaStream_t st);

// Accumulates into m.grad the gradient of the mean squared error over the examples
// `idx` (or 0..n_ex-1 when idx is NULL) and adds the summed squared error to m.loss.
Status mlp_grad(Mlp& m, const float* F, const float* T, const int64_t* idx, int64_t n_ex,
                cudaStream_t st);

// steps Adam steps (lr, betas 0.9/0.999) on mini-batches of `batch` examples drawn
// from the training examples (every example whose sample index i = e % n has
// i % holdout != 0).  The steps run as launches of one captured CUDA graph of up to
// 25 steps, kept in m and reused while F, T and the sizes stay the same.
Status mlp_train(Mlp& m, const float* F, const float* T, int64_t n, int q, int steps, int batch,
                 float lr, int holdout, cudaStream_t st);

// Mean squared error and the mean squared target over the held-out examples
// (sample index i % holdout == 0).
Status mlp_validate(Mlp& m, const float* F, const float* T, int64_t n, int q, int holdout,
                    double* mse, double* target_ms, cudaStream_t st);

}  // namespace saige
