// FP64 vector kernels of the PCG and AI-REML loops.  Vectors of a block are
// stored column after column with leading dimension ld (>= n).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace saige {

// Per-column PCG state kept on the device.
enum : int32_t { kColActive = 0, kColConverged = 1, kColStopped = 2, kColMaxIter = 3 };

struct PcgCols {
  double* rz;       // r'z
  double* rr;       // r'r
  double* pap;      // p'Ap
  double* tol_abs;  // tol * max(||b||, 1)
  int32_t* state;   // kCol*
  int32_t* iters;
};

// Number of partial-sum blocks used by the reductions below.
int red_blocks(int64_t n);

// out[c] = sum_i a[i,c] * b[i,c] for c < q (two-stage, fixed order).
// partial must hold red_blocks(n) * q doubles.
cudaError_t col_dots(const double* a, const double* b, int64_t n, int64_t ld, int q,
                     double* partial, double* out, cudaStream_t st);

// D (p x q, row-major) = A' diag(w) B, A: n x p, B: n x q (w may be NULL).
// partial must hold red_blocks(n) * p * q doubles.
cudaError_t cross_dots(const double* a, int p, const double* b, int q, const double* w, int64_t n,
                       int64_t ld, double* partial, double* out, cudaStream_t st);

// PCG building blocks (columns with state != active are left untouched).
// Start: x = x0 (or 0), r = b - ax0 (ax0 may be NULL meaning A x0 = 0),
// z = r / d, p = z; rz, rr and tol_abs per column; state = active, or
// converged when ||r|| < tol_abs already (unless force_step).
cudaError_t pcg_start(const double* b, const double* x0, const double* ax0, const double* d,
                      double* x, double* r, double* z, double* p, int64_t n, int64_t ld, int q,
                      double tol, bool force_step, PcgCols cols, double* partial,
                      double* scratch3q, cudaStream_t st);
// ap = tau0 p / wmax + tau1 kp, pap = p'ap; columns with |pap| < 1e-30 stop.
cudaError_t pcg_apply(const double* p, const double* kp, const double* wmax, double tau0,
                      double tau1, double* ap, int64_t n, int64_t ld, int q, PcgCols cols,
                      double* partial, cudaStream_t st);
// Variant for the score-test convention: ap = tau0 w p + tau1 kp.
cudaError_t pcg_apply_w(const double* p, const double* kp, const double* w, double tau0,
                        double tau1, double* ap, int64_t n, int64_t ld, int q, PcgCols cols,
                        double* partial, cudaStream_t st);
// x += alpha p, r -= alpha ap, z = r / d, then beta, ||r|| test, p = z + beta p;
// with kx, also kx += alpha kp (K x kept beside x from the products K p).
cudaError_t pcg_step(double* x, double* r, double* z, double* p, const double* ap,
                     const double* d, int64_t n, int64_t ld, int q, int max_iter, PcgCols cols,
                     double* partial, double* scratch2q, cudaStream_t st, double* kx = nullptr,
                     const double* kp = nullptr);

// Elementwise helpers for the AI-REML loop.
// Jacobi diagonal of fit-null: wmax = max(w,1e-30), d = tau0/wmax + tau1 (1 when |d| <= 1e-30);
// with diagk, d = tau0/wmax + tau1 diagk[i].
cudaError_t sigma_diag(const double* w, double tau0, double tau1, double* wmax, double* d,
                       int64_t n, cudaStream_t st, const double* diagk = nullptr);
// Jacobi diagonal of solve_mixed_model_pcg: d = tau0 w + tau1.
cudaError_t sigma_diag_w(const double* w, double tau0, double tau1, double* d, int64_t n,
                         cudaStream_t st);
// eta = X alpha, mu = g^-1(eta) clamped (family.rs:82-90).
cudaError_t eta_mu(const double* x, int p, const double* alpha, int trait, double* eta, double* mu,
                   int64_t n, int64_t ld, cudaStream_t st);
// w = max(V(mu),1e-30), ytil = eta + (y-mu)/max(w,1e-30)  (family.rs:55-66, ai_reml.rs:168-173)
cudaError_t work_vectors(const double* y, const double* eta, const double* mu, int trait,
                         double* w, double* ytil, int64_t n, cudaStream_t st);
// mu = initialize_mu(y), eta = link(mu)  (family.rs:23-45)
cudaError_t init_mu(const double* y, int trait, double* mu, double* eta, int64_t n,
                    cudaStream_t st);
// Y[:,c] -= sum_j A[:,j] coef[j*q + c]   (A: n x p, Y: n x q)
cudaError_t sub_combo(double* y, int q, const double* a, int p, const double* coef, int64_t n,
                      int64_t ld, cudaStream_t st);
// out = v / max(w,1e-30)
cudaError_t div_w(const double* v, const double* w, double* out, int64_t n, cudaStream_t st);
// nrv Rademacher probe columns (ld apart, padding rows zeroed) from the ChaCha8
// stream with the given key (ai_reml.rs:121-130).
cudaError_t rademacher_probes_dev(const uint32_t* key, double* out, int64_t n, int64_t ld, int nrv,
                                  cudaStream_t st);
// Rows m with excl[m] != 0 set to zero in q columns (ld apart): markers left out of
// a leave-one-chromosome-out product.
cudaError_t mask_rows_f64(double* u, int64_t ld, int q, const uint8_t* excl, int64_t m,
                          cudaStream_t st);
cudaError_t mask_rows_f32(float* u, const uint8_t* excl, int64_t m, cudaStream_t st);
cudaError_t zero_pad(double* v, int64_t n, int64_t ld, int q, cudaStream_t st);

}  // namespace saige
