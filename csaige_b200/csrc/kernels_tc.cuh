// Tensor-core (tcgen05, kind::i8) GRM product: the MIXED precision path.
#pragma once
#include "engine.cuh"

namespace saige {

// Columns of one tensor-core launch that keep its fastest ring shape: with 3 r limb
// columns rounded up to 16 at most 128, the two accumulators leave the TMEM room for
// four operand slots and pass B's load stages of two sub-stages fit three deep (43
// columns take 144 MMA columns: two slots and a slower shape).
constexpr int kTcFastCols = 42;

// Kv for q columns (ld = h->n_pad) through the int8-limb tensor-core kernels.
Status tc_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                  cudaStream_t st);
void tc_destroy(saige_grm* h);
// Streamed build: reserves the code tiles for up to rows_cap marker rows (the
// sample-major tiles keep that many marker tiles per sample tile), then builds the
// tiles of marker tiles [mt0, mt1) from h->geno as those rows are complete.
Status tc_stream_begin(saige_grm* h, int64_t rows_cap);
Status tc_stream_tiles(saige_grm* h, int64_t mt0, int64_t mt1, cudaStream_t st);
// Missing calls in the handle's lists for one-column products (-1: none built, or declined).
int64_t tc_missing_listed(const saige_grm* h);
// Trial launches the ring-shape autotuner has timed in this process.
int64_t tc_autotune_trials();
// Budget of every pipeline wait of the tensor-core product, in SM cycles (< 0: the
// default, ~2 s); 0 makes a wait that is not already satisfied give up at once.
void tc_set_wait_budget(long long cycles);

}  // namespace saige
