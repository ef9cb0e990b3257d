// FP64 vector kernels for the PCG recurrence (saige-linalg/src/
// decomposition.rs:212-298), the fit-null operator and Jacobi preconditioner
// (saige-core/src/glmm/ai_reml.rs:142-164) and the AI-REML elementwise work
// (family.rs, link.rs).  Reductions are two-stage with a partition fixed by n,
// so every result is deterministic from run to run.
#include <math.h>

#include "common.cuh"
#include "kernels_vec.cuh"
#include "rng.hpp"

namespace saige {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int k = 0; k < kT / 32; ++k) s += sh[k];
  }
  __syncthreads();
  return s;  // valid in thread 0
}

__device__ __forceinline__ int64_t part_chunk(int64_t n) {
  return (n + gridDim.x - 1) / gridDim.x;
}

// Sum nb partials of k quantities per column in a fixed order; one warp per
// (column, quantity).
__global__ void reduce_partials(const double* __restrict__ partial, int nb, int nq,
                                double* __restrict__ out) {
  const int idx = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (idx >= nq) return;
  const int l = threadIdx.x & 31;
  double s = 0.0;
  for (int b = l; b < nb; b += 32) s += partial[(int64_t)idx * nb + b];
  s = warp_sum(s);
  if (l == 0) out[idx] = s;
}

__global__ void col_dots_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                int64_t n, int64_t ld, double* __restrict__ partial) {
  __shared__ double sh[kT / 32];
  const int c = blockIdx.y;
  const int64_t ch = part_chunk(n), lo = (int64_t)blockIdx.x * ch;
  int64_t hi = lo + ch;
  if (hi > n) hi = n;
  const double* ac = a + (int64_t)c * ld;
  const double* bc = b + (int64_t)c * ld;
  double s = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kT) s += ac[i] * bc[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partial[(int64_t)c * gridDim.x + blockIdx.x] = s;
}

__global__ void cross_dots_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                  int q, const double* __restrict__ w, int64_t n, int64_t ld,
                                  double* __restrict__ partial) {
  __shared__ double sh[kT / 32];
  const int pair = blockIdx.y;
  const int j = pair / q, k = pair % q;
  const int64_t ch = part_chunk(n), lo = (int64_t)blockIdx.x * ch;
  int64_t hi = lo + ch;
  if (hi > n) hi = n;
  const double* aj = a + (int64_t)j * ld;
  const double* bk = b + (int64_t)k * ld;
  double s = 0.0;
  if (w) {
    for (int64_t i = lo + threadIdx.x; i < hi; i += kT) s += aj[i] * w[i] * bk[i];
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += kT) s += aj[i] * bk[i];
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partial[(int64_t)pair * gridDim.x + blockIdx.x] = s;
}

__global__ void pcg_start_kernel(const double* __restrict__ b, const double* __restrict__ x0,
                                 const double* __restrict__ ax0, const double* __restrict__ d,
                                 double* __restrict__ x, double* __restrict__ r,
                                 double* __restrict__ z, double* __restrict__ p, int64_t n,
                                 int64_t ld, double* __restrict__ partial) {
  __shared__ double sh[kT / 32];
  const int c = blockIdx.y;
  const int64_t off = (int64_t)c * ld;
  const int64_t ch = part_chunk(n), lo = (int64_t)blockIdx.x * ch;
  int64_t hi = lo + ch;
  if (hi > n) hi = n;
  double s_rz = 0.0, s_rr = 0.0, s_bb = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kT) {
    const double bi = b[off + i];
    const double xi = x0 ? x0[off + i] : 0.0;
    const double ri = bi - (ax0 ? ax0[off + i] : 0.0);
    const double zi = ri / d[i];
    x[off + i] = xi;
    r[off + i] = ri;
    z[off + i] = zi;
    p[off + i] = zi;
    s_rz += ri * zi;
    s_rr += ri * ri;
    s_bb += bi * bi;
  }
  const int nb = gridDim.x, q = gridDim.y;
  s_rz = block_sum(s_rz, sh);
  s_rr = block_sum(s_rr, sh);
  s_bb = block_sum(s_bb, sh);
  if (threadIdx.x == 0) {
    partial[((int64_t)0 * q + c) * nb + blockIdx.x] = s_rz;
    partial[((int64_t)1 * q + c) * nb + blockIdx.x] = s_rr;
    partial[((int64_t)2 * q + c) * nb + blockIdx.x] = s_bb;
  }
}

__global__ void pcg_start_finish(const double* __restrict__ sums, int q, double tol, int force_step,
                                 PcgCols cols) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= q) return;
  const double rz = sums[c], rr = sums[q + c], bb = sums[2 * q + c];
  const double bn = sqrt(bb);
  const double tol_abs = tol * (bn > 1.0 ? bn : 1.0);
  cols.rz[c] = rz;
  cols.rr[c] = rr;
  cols.tol_abs[c] = tol_abs;
  cols.iters[c] = 0;
  // a warm-started column takes at least one CG step (force_step), so a start
  // that already meets the tolerance is still refined against the current operator
  cols.state[c] = (!force_step && sqrt(rr) < tol_abs) ? kColConverged : kColActive;
}

template <bool kWInverse>
__global__ void pcg_apply_kernel(const double* __restrict__ p, const double* __restrict__ kp,
                                 const double* __restrict__ wv, double tau0, double tau1,
                                 double* __restrict__ ap, int64_t n, int64_t ld,
                                 const int32_t* __restrict__ state, double* __restrict__ partial) {
  __shared__ double sh[kT / 32];
  const int c = blockIdx.y;
  if (state[c] != kColActive) return;
  const int64_t off = (int64_t)c * ld;
  const int64_t ch = part_chunk(n), lo = (int64_t)blockIdx.x * ch;
  int64_t hi = lo + ch;
  if (hi > n) hi = n;
  double s = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kT) {
    const double pi = p[off + i];
    // ai_reml.rs:147 (tau0 v / max(w,1e-30) + tau1 Kv) or pcg.rs:56 (tau0 w v + tau1 Kv)
    const double a = kWInverse ? tau0 * pi / wv[i] + tau1 * kp[off + i]
                               : tau0 * wv[i] * pi + tau1 * kp[off + i];
    ap[off + i] = a;
    s += pi * a;
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) partial[(int64_t)c * gridDim.x + blockIdx.x] = s;
}

__global__ void pcg_apply_finish(const double* __restrict__ partial, int nb, int q, PcgCols cols) {
  const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (c >= q) return;
  if (cols.state[c] != kColActive) return;
  const int l = threadIdx.x & 31;
  double s = 0.0;
  for (int b = l; b < nb; b += 32) s += partial[(int64_t)c * nb + b];
  s = warp_sum(s);
  if (l == 0) {
    cols.pap[c] = s;
    if (fabs(s) < 1e-30) cols.state[c] = kColStopped;  // decomposition.rs:257-264
  }
}

__global__ void pcg_update_kernel(double* __restrict__ x, double* __restrict__ r,
                                  double* __restrict__ z, const double* __restrict__ p,
                                  const double* __restrict__ ap, const double* __restrict__ d,
                                  int64_t n, int64_t ld, PcgCols cols,
                                  double* __restrict__ partial, double* __restrict__ kx,
                                  const double* __restrict__ kp) {
  __shared__ double sh[kT / 32];
  const int c = blockIdx.y;
  if (cols.state[c] != kColActive) return;
  const double alpha = cols.rz[c] / cols.pap[c];
  const int64_t off = (int64_t)c * ld;
  const int64_t ch = part_chunk(n), lo = (int64_t)blockIdx.x * ch;
  int64_t hi = lo + ch;
  if (hi > n) hi = n;
  double s_rz = 0.0, s_rr = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kT) {
    x[off + i] += alpha * p[off + i];
    if (kx) kx[off + i] += alpha * kp[off + i];  // K x follows x: K x += alpha K p
    const double ri = r[off + i] - alpha * ap[off + i];
    r[off + i] = ri;
    const double zi = ri / d[i];
    z[off + i] = zi;
    s_rz += ri * zi;
    s_rr += ri * ri;
  }
  const int nb = gridDim.x, q = gridDim.y;
  s_rz = block_sum(s_rz, sh);
  s_rr = block_sum(s_rr, sh);
  if (threadIdx.x == 0) {
    partial[((int64_t)0 * q + c) * nb + blockIdx.x] = s_rz;
    partial[((int64_t)1 * q + c) * nb + blockIdx.x] = s_rr;
  }
}

__global__ void pcg_update_finish(const double* __restrict__ partial, int nb, int q,
                                  int max_iter, PcgCols cols, double* __restrict__ beta) {
  const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (c >= q) return;
  if (cols.state[c] != kColActive) return;
  const int l = threadIdx.x & 31;
  double s_rz = 0.0, s_rr = 0.0;
  for (int b = l; b < nb; b += 32) {
    s_rz += partial[((int64_t)0 * q + c) * nb + b];
    s_rr += partial[((int64_t)1 * q + c) * nb + b];
  }
  s_rz = warp_sum(s_rz);
  s_rr = warp_sum(s_rr);
  if (l == 0) {
    beta[c] = s_rz / cols.rz[c];
    cols.rz[c] = s_rz;
    cols.rr[c] = s_rr;
    const int it = cols.iters[c] + 1;
    cols.iters[c] = it;
    if (sqrt(s_rr) < cols.tol_abs[c]) cols.state[c] = kColConverged;
    else if (it >= max_iter) cols.state[c] = kColMaxIter;
  }
}

__global__ void pcg_p_kernel(double* __restrict__ p, const double* __restrict__ z, int64_t n,
                             int64_t ld, const int32_t* __restrict__ state,
                             const double* __restrict__ beta) {
  const int c = blockIdx.y;
  if (state[c] != kColActive) return;
  const double bt = beta[c];
  const int64_t off = (int64_t)c * ld;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[off + i] = z[off + i] + bt * p[off + i];
}

__global__ void sigma_diag_kernel(const double* __restrict__ w, double tau0, double tau1,
                                  const double* __restrict__ diagk, double* __restrict__ wmax,
                                  double* __restrict__ d, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double wm = w[i] > 1e-30 ? w[i] : 1e-30;
  const double dg = diagk ? tau0 / wm + tau1 * diagk[i] : tau0 / wm + tau1;
  wmax[i] = wm;
  d[i] = fabs(dg) > 1e-30 ? dg : 1.0;
}

__global__ void sigma_diag_w_kernel(const double* __restrict__ w, double tau0, double tau1,
                                    double* __restrict__ d, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double dg = tau0 * w[i] + tau1;
  d[i] = fabs(dg) > 1e-30 ? dg : 1.0;
}

__device__ __forceinline__ double inv_link(int t, double eta) {
  if (t == SAIGE_TRAIT_BINARY) return 1.0 / (1.0 + exp(-eta));
  if (t == SAIGE_TRAIT_QUANTITATIVE) return eta;
  return 1.0 - exp(-exp(eta));
}

__global__ void eta_mu_kernel(const double* __restrict__ x, int p, const double* __restrict__ alpha,
                              int t, double* __restrict__ eta, double* __restrict__ mu, int64_t n,
                              int64_t ld) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // DenseMatrix::mat_vec column sweep order (dense.rs:102-113)
  double e = 0.0;
  for (int j = 0; j < p; ++j) e += x[(int64_t)j * ld + i] * alpha[j];
  eta[i] = e;
  double m = inv_link(t, e);
  if (t != SAIGE_TRAIT_QUANTITATIVE) {
    if (m < 1e-10) m = 1e-10;
    if (m > 1.0 - 1e-10) m = 1.0 - 1e-10;
  }
  mu[i] = m;
}

__global__ void work_vectors_kernel(const double* __restrict__ y, const double* __restrict__ eta,
                                    const double* __restrict__ mu, int t, double* __restrict__ w,
                                    double* __restrict__ ytil, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double m = mu[i];
  double v = t == SAIGE_TRAIT_QUANTITATIVE ? 1.0 : m * (1.0 - m);
  v = v > 1e-30 ? v : 1e-30;
  w[i] = v;
  if (ytil) {
    const double wm = v > 1e-30 ? v : 1e-30;
    ytil[i] = eta[i] + (y[i] - m) / wm;
  }
}

__global__ void init_mu_kernel(const double* __restrict__ y, int t, double* __restrict__ mu,
                               double* __restrict__ eta, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double yi = y[i];
  double m, e;
  if (t == SAIGE_TRAIT_BINARY) {
    m = (yi + 0.5) / 2.0;
    e = log(m / (1.0 - m));
  } else if (t == SAIGE_TRAIT_QUANTITATIVE) {
    m = yi;
    e = m;
  } else {
    m = (yi + 0.5) / 2.0;
    m = m < 0.01 ? 0.01 : (m > 0.99 ? 0.99 : m);
    e = log(-log(1.0 - m));
  }
  mu[i] = m;
  eta[i] = e;
}

__global__ void sub_combo_kernel(double* __restrict__ y, int q, const double* __restrict__ a,
                                 int p, const double* __restrict__ coef, int64_t n, int64_t ld) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = y[(int64_t)c * ld + i];
  // ai_reml.rs:247-251: one subtraction per covariate column, in order
  for (int j = 0; j < p; ++j) v -= a[(int64_t)j * ld + i] * coef[j * q + c];
  y[(int64_t)c * ld + i] = v;
}

__global__ void div_w_kernel(const double* __restrict__ v, const double* __restrict__ w,
                             double* __restrict__ out, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double wm = w[i] > 1e-30 ? w[i] : 1e-30;
  out[i] = v[i] / wm;
}

struct Key8 {
  uint32_t w[8];
};

// Rademacher probes from the ChaCha8 stream: word k = r * n + i (one block of 16
// words per thread) gives column r, sample i the value +1 when its sign bit is set
// (rand's gen::<bool>), else -1; rows n .. ld-1 of every column are zeroed.
__global__ void rademacher_kernel(Key8 key, int64_t n, int64_t ld, int nrv, double* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t words = (int64_t)nrv * n;
  if (c * 16 < words) {
    uint32_t w[16];
    chacha8_block(key.w, (uint64_t)c, w);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int64_t k = c * 16 + j;
      if (k < words) {
        const int64_t r = k / n, i = k - r * n;
        out[r * ld + i] = static_cast<int32_t>(w[j]) < 0 ? 1.0 : -1.0;
      }
    }
  }
  // padding rows (ld - n per column)
  const int64_t pad = (ld - n) * nrv;
  for (int64_t e = c; e < pad; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = e / (ld - n), i = n + (e - r * (ld - n));
    out[r * ld + i] = 0.0;
  }
}

template <class T>
__global__ void mask_rows_kernel(T* __restrict__ u, int64_t ld, const uint8_t* __restrict__ excl,
                                 int64_t m) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m && excl[i]) u[(int64_t)c * ld + i] = T(0);
}

__global__ void zero_pad_kernel(double* __restrict__ v, int64_t n, int64_t ld) {
  const int c = blockIdx.y;
  const int64_t i = n + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ld) v[(int64_t)c * ld + i] = 0.0;
}

inline unsigned g1(int64_t n) { return (unsigned)ceil_div(n, kT); }

}  // namespace

int red_blocks(int64_t n) {
  int64_t b = ceil_div(n, 4096);
  if (b < 1) b = 1;
  if (b > 256) b = 256;
  return (int)b;
}

cudaError_t col_dots(const double* a, const double* b, int64_t n, int64_t ld, int q,
                     double* partial, double* out, cudaStream_t st) {
  const int nb = red_blocks(n);
  col_dots_kernel<<<dim3(nb, q), kT, 0, st>>>(a, b, n, ld, partial);
  reduce_partials<<<(unsigned)ceil_div(q, 8), 256, 0, st>>>(partial, nb, q, out);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t cross_dots(const double* a, int p, const double* b, int q, const double* w, int64_t n,
                       int64_t ld, double* partial, double* out, cudaStream_t st) {
  const int nb = red_blocks(n);
  cross_dots_kernel<<<dim3(nb, p * q), kT, 0, st>>>(a, b, q, w, n, ld, partial);
  reduce_partials<<<(unsigned)ceil_div(p * q, 8), 256, 0, st>>>(partial, nb, p * q, out);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t pcg_start(const double* b, const double* x0, const double* ax0, const double* d,
                      double* x, double* r, double* z, double* p, int64_t n, int64_t ld, int q,
                      double tol, bool force_step, PcgCols cols, double* partial,
                      double* scratch3q, cudaStream_t st) {
  const int nb = red_blocks(n);
  pcg_start_kernel<<<dim3(nb, q), kT, 0, st>>>(b, x0, ax0, d, x, r, z, p, n, ld, partial);
  reduce_partials<<<(unsigned)ceil_div(3 * q, 8), 256, 0, st>>>(partial, nb, 3 * q, scratch3q);
  pcg_start_finish<<<(unsigned)ceil_div(q, 64), 64, 0, st>>>(scratch3q, q, tol, force_step ? 1 : 0,
                                                             cols);
  count_launches(3);
  return cudaGetLastError();
}

cudaError_t pcg_apply(const double* p, const double* kp, const double* wmax, double tau0,
                      double tau1, double* ap, int64_t n, int64_t ld, int q, PcgCols cols,
                      double* partial, cudaStream_t st) {
  const int nb = red_blocks(n);
  pcg_apply_kernel<true><<<dim3(nb, q), kT, 0, st>>>(p, kp, wmax, tau0, tau1, ap, n, ld,
                                                     cols.state, partial);
  pcg_apply_finish<<<(unsigned)ceil_div(q, 8), 256, 0, st>>>(partial, nb, q, cols);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t pcg_apply_w(const double* p, const double* kp, const double* w, double tau0,
                        double tau1, double* ap, int64_t n, int64_t ld, int q, PcgCols cols,
                        double* partial, cudaStream_t st) {
  const int nb = red_blocks(n);
  pcg_apply_kernel<false><<<dim3(nb, q), kT, 0, st>>>(p, kp, w, tau0, tau1, ap, n, ld,
                                                      cols.state, partial);
  pcg_apply_finish<<<(unsigned)ceil_div(q, 8), 256, 0, st>>>(partial, nb, q, cols);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t pcg_step(double* x, double* r, double* z, double* p, const double* ap,
                     const double* d, int64_t n, int64_t ld, int q, int max_iter, PcgCols cols,
                     double* partial, double* scratch2q, cudaStream_t st, double* kx, const double* kp) {
  const int nb = red_blocks(n);
  pcg_update_kernel<<<dim3(nb, q), kT, 0, st>>>(x, r, z, p, ap, d, n, ld, cols, partial, kx, kp);
  pcg_update_finish<<<(unsigned)ceil_div(q, 8), 256, 0, st>>>(partial, nb, q, max_iter, cols,
                                                              scratch2q);
  unsigned gx = (unsigned)ceil_div(n, kT);
  if (gx > 1024) gx = 1024;
  pcg_p_kernel<<<dim3(gx, q), kT, 0, st>>>(p, z, n, ld, cols.state, scratch2q);
  count_launches(3);
  return cudaGetLastError();
}

cudaError_t sigma_diag(const double* w, double tau0, double tau1, double* wmax, double* d,
                       int64_t n, cudaStream_t st, const double* diagk) {
  sigma_diag_kernel<<<g1(n), kT, 0, st>>>(w, tau0, tau1, diagk, wmax, d, n);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t sigma_diag_w(const double* w, double tau0, double tau1, double* d, int64_t n,
                         cudaStream_t st) {
  sigma_diag_w_kernel<<<g1(n), kT, 0, st>>>(w, tau0, tau1, d, n);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t eta_mu(const double* x, int p, const double* alpha, int trait, double* eta, double* mu,
                   int64_t n, int64_t ld, cudaStream_t st) {
  eta_mu_kernel<<<g1(n), kT, 0, st>>>(x, p, alpha, trait, eta, mu, n, ld);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t work_vectors(const double* y, const double* eta, const double* mu, int trait,
                         double* w, double* ytil, int64_t n, cudaStream_t st) {
  work_vectors_kernel<<<g1(n), kT, 0, st>>>(y, eta, mu, trait, w, ytil, n);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t init_mu(const double* y, int trait, double* mu, double* eta, int64_t n,
                    cudaStream_t st) {
  init_mu_kernel<<<g1(n), kT, 0, st>>>(y, trait, mu, eta, n);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t sub_combo(double* y, int q, const double* a, int p, const double* coef, int64_t n,
                      int64_t ld, cudaStream_t st) {
  sub_combo_kernel<<<dim3(g1(n), q), kT, 0, st>>>(y, q, a, p, coef, n, ld);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t div_w(const double* v, const double* w, double* out, int64_t n, cudaStream_t st) {
  div_w_kernel<<<g1(n), kT, 0, st>>>(v, w, out, n);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t rademacher_probes_dev(const uint32_t* key, double* out, int64_t n, int64_t ld, int nrv,
                                  cudaStream_t st) {
  Key8 k;
  for (int i = 0; i < 8; ++i) k.w[i] = key[i];
  const int64_t blocks = ceil_div((int64_t)nrv * n, 16);
  const int64_t pad = (ld - n) * nrv;
  const int64_t threads = blocks > pad ? blocks : pad;
  rademacher_kernel<<<(unsigned)ceil_div(threads > 0 ? threads : 1, kT), kT, 0, st>>>(k, n, ld, nrv, out);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t mask_rows_f64(double* u, int64_t ld, int q, const uint8_t* excl, int64_t m,
                          cudaStream_t st) {
  mask_rows_kernel<double><<<dim3(g1(m), q), kT, 0, st>>>(u, ld, excl, m);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t mask_rows_f32(float* u, const uint8_t* excl, int64_t m, cudaStream_t st) {
  mask_rows_kernel<float><<<dim3(g1(m), 1), kT, 0, st>>>(u, m, excl, m);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t zero_pad(double* v, int64_t n, int64_t ld, int q, cudaStream_t st) {
  if (ld <= n) return cudaSuccess;
  zero_pad_kernel<<<dim3(g1(ld - n), q), kT, 0, st>>>(v, n, ld);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace saige
