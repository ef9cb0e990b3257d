// Warm starts for the PCG solves of AI-REML: the recycled (Galerkin) start, the
// learned correction (a small MLP) and diag(K).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

struct saige_grm;

namespace saige {

// D (a x b, row-major) = A' B over n rows; A: a columns and B: b columns, ld apart.
// Each block sums a fixed row chunk; the chunks are then added in order, so the
// result does not depend on scheduling.  partial: gram_partial_doubles(n, a, b).
size_t gram_partial_doubles(int64_t n, int a, int b);
cudaError_t gram(const double* A, int a, const double* B, int b, int64_t n, int64_t ld,
                 double* partial, double* out, cudaStream_t st);

// Y[:, c] (c < q) = sum_{j < m} V[:, j] G[j*q + c]  (+ Y[:, c] when add); G on the device.
// Y must not overlap V.  Rows n .. ld-1 are not written.
cudaError_t combo(const double* V, int m, const double* G, int q, double* Y, bool add, int64_t n,
                  int64_t ld, cudaStream_t st);

// out[:, c] = tau0 v[:, c] / wmax + tau1 kv[:, c]  (the fit-null Sigma applied to v given K v)
cudaError_t sigma_image(const double* v, const double* kv, const double* wmax, double tau0,
                        double tau1, double* out, int64_t n, int64_t ld, int q, cudaStream_t st);

// out[:, c] = a[:, c] - b[:, c]
cudaError_t sub_cols(const double* a, const double* b, double* out, int64_t n, int64_t ld, int q,
                     cudaStream_t st);

// Learned start: features of example e = c * n + i (sample i, column c) for the
// prediction of the next solution change, 16 floats each:
//   x[i,c] / sx[c], b[i,c] / sb[c], (bnext[i,c] - b[i,c]) / sb[c], log(wnext[i] / w[i]),
//   d[i] / dmean - 1, diagk[i] - 1, the sketches ku[i, s] / sk[s] for s < n_sk (the GRM
//   applied to the first n_sk <= 8 probes; zero past n_sk), tau1, 0
// (x, b, bnext, ku: ld apart; d the Jacobi scale 1 / (tau0 / w + tau1); scales =
// [sx (q), sb (q), sk (8)]).
cudaError_t learn_features(const double* x, const double* b, const double* bnext, const double* w,
                           const double* wnext, const double* diagk, const double* ku, int n_sk,
                           const double* scales, double tau0, double tau1, double dmean,
                           int64_t n, int64_t ld, int q, float* F, cudaStream_t st);
// T[c*n + i] = (x1[i,c] - x0[i,c]) / s[c]
cudaError_t learn_targets(const double* x1, const double* x0, const double* s, int64_t n,
                          int64_t ld, int q, float* T, cudaStream_t st);
// out[:, c] = y[c*n + i] (double columns, ld apart; padding rows left as they are)
cudaError_t learn_to_cols(const float* y, int64_t n, int64_t ld, int q, double* out,
                          cudaStream_t st);

// diag K (n values): (1/M') sum over the markers in the product (the LOCO mask
// honoured) of z_im^2, z from the handle's 2p and 1/s in f64 (K8; the diagonal
// SAIGE's C++ computes in Get_Diagof_StdGeno).
Status grm_diag(saige_grm* h, double* out, cudaStream_t st);

}  // namespace saige
