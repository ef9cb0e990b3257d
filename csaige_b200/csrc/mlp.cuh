// The learned part of the PCG warm start: an MLP of 16 inputs, three tanh layers of
// 256 units and one linear output, with BF16 weights and BF16 activations (FP32
// arithmetic and FP32 master weights), trained on the GPU by this library's own
// kernels.  The two 256 x 256 layers of the forward pass run on the tensor cores
// (tcgen05.mma kind::f16, A and B from shared memory, FP32 accumulators in tensor
// memory, the bias, tanh and BF16 rounding fused into the epilogue); the input layer,
// the backward pass (blocked FP32 GEMMs with a fixed summation order) and Adam run on
// the CUDA cores.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "engine.cuh"

namespace saige {

constexpr int kMlpIn = 16;
constexpr int kMlpH = 256;
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

// Examples of one training mini-batch (a multiple of 128).
constexpr int kMlpBatch = 8192;

struct Mlp {
  DevBuf mem;                 // master, grad, Adam moments, loss, step, BF16 copy
  DevBuf wimg;                // W2 and W3 as BF16 B-operand images (2 x 128 KB)
  DevBuf work;                // activations and images of one chunk of examples
  size_t work_rows = 0;       // examples the work buffer holds (multiple of 128)
  DevBuf gpart;               // split-K partials of the weight gradients
  cudaGraphExec_t graph = nullptr;  // captured training steps (see mlp_train)
  const void* graph_key[2] = {nullptr, nullptr};
  int64_t graph_n = 0;
  int graph_q = 0, graph_holdout = 0, graph_steps = 0;
  float graph_lr = 0.f;
  ~Mlp() {
    if (graph) cudaGraphExecDestroy(graph);
  }
  float* master = nullptr;    // FP32 weights
  uint16_t* wbf = nullptr;    // BF16 copy used by the forward pass
  float* grad = nullptr;      // gradient of the last pass
  float* m1 = nullptr;        // Adam moments
  float* m2 = nullptr;
  int* step = nullptr;        // device step counter (mini-batch offset, Adam bias correction)
  double* loss = nullptr;     // [2]: summed squared error of the last pass, example count
  unsigned int* err = nullptr;  // a tensor-core layer's pipeline wait ran out (nonzero)
  bool ready = false;         // initialised
  int64_t trained_steps = 0;
};

// Allocates and initialises the weights (uniform +-1/sqrt(fan_in), from seed).
Status mlp_init(Mlp& m, uint64_t seed, cudaStream_t st);

// out[e] = MLP(F[e*16 .. e*16+16]) for e < n_ex.
Status mlp_forward(Mlp& m, const float* F, int64_t n_ex, float* out, cudaStream_t st);

// m.grad = the gradient of the mean squared error over the examples 0..n_ex-1 (with
// respect to the FP32 master weights, through the BF16 roundings), m.loss[0] = the
// summed squared error.
Status mlp_grad(Mlp& m, const float* F, const float* T, int64_t n_ex, cudaStream_t st);

// steps Adam steps (lr, betas 0.9/0.999) on mini-batches of kMlpBatch examples drawn
// from the training examples (every example whose sample index i = e % n has
// i % holdout != 0).  The steps run as launches of one captured CUDA graph of up to
// 25 steps, kept in m and reused while F, T and the sizes stay the same.
Status mlp_train(Mlp& m, const float* F, const float* T, int64_t n, int q, int steps, float lr,
                 int holdout, cudaStream_t st);

// Mean squared error and the mean squared target over the held-out examples
// (sample index i % holdout == 0).
Status mlp_validate(Mlp& m, const float* F, const float* T, int64_t n, int q, int holdout,
                    double* mse, double* target_ms, cudaStream_t st);

}  // namespace saige
