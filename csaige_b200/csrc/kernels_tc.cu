// Tensor-core GRM product (MIXED precision) — not built yet.
#include "kernels_tc.cuh"

namespace saige {

Status tc_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                  cudaStream_t st) {
  (void)h; (void)v; (void)kp; (void)q; (void)active; (void)st;
  return fail(SAIGE_ENOTSUP, "MIXED precision is not available in this build");
}

void tc_destroy(saige_grm* h) { (void)h; }

}  // namespace saige
