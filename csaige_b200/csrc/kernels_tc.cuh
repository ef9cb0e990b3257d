// Tensor-core (tcgen05, kind::i8) GRM product: the MIXED precision path.
#pragma once
#include "engine.cuh"

namespace saige {

// Kv for q columns (ld = h->n_pad) through the int8-limb tensor-core kernels.
Status tc_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                  cudaStream_t st);
void tc_destroy(saige_grm* h);
// Trial launches the ring-shape autotuner has timed in this process.
int64_t tc_autotune_trials();

}  // namespace saige
