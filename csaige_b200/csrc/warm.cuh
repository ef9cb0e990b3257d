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

// diag K (n values): (1/M') sum over the markers in the product (the LOCO mask
// honoured) of z_im^2, z from the handle's 2p and 1/s in f64 (K8; the diagonal
// SAIGE's C++ computes in Get_Diagof_StdGeno).
Status grm_diag(saige_grm* h, double* out, cudaStream_t st);

}  // namespace saige
