// Building blocks of the recycled PCG start (Galerkin projection onto vectors
// whose Sigma-image is known without a GRM product) and diag(K).
#include <algorithm>

#include "engine.cuh"
#include "warm.cuh"

namespace saige {
namespace {

constexpr int kG = 32;        // Gram tile (32 x 32 outputs per block)
constexpr int kGThreads = 256;

int gram_chunks(int64_t n, int a, int b) {
  const int tiles = ((a + kG - 1) / kG) * ((b + kG - 1) / kG);
  const int64_t by_rows = (n + 2047) / 2048;
  const int64_t want = std::max<int64_t>(1, 148 * 4 / std::max(tiles, 1));
  return (int)std::max<int64_t>(1, std::min(by_rows, want));
}

// Block (chunk x, tile y): rows [x*chunk, (x+1)*chunk) of the 32 x 32 output tile y.
__global__ void __launch_bounds__(kGThreads)
    gram_kernel(const double* __restrict__ A, int a, const double* __restrict__ B, int b,
                int64_t n, int64_t ld, int64_t chunk, double* __restrict__ partial) {
  __shared__ double as[kG][kG + 1], bs[kG][kG + 1];
  const int tiles_b = (b + kG - 1) / kG;
  const int ta = blockIdx.y / tiles_b, tb = blockIdx.y % tiles_b;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // ty 0..7
  const int64_t lo = (int64_t)blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t r0 = lo; r0 < hi; r0 += kG) {
    const int64_t row = r0 + tx;
#pragma unroll
    for (int k = ty; k < kG; k += 8) {
      const int ca = ta * kG + k, cb = tb * kG + k;
      as[tx][k] = (ca < a && row < hi) ? A[(int64_t)ca * ld + row] : 0.0;
      bs[tx][k] = (cb < b && row < hi) ? B[(int64_t)cb * ld + row] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int r = 0; r < kG; ++r) {
      const double bv = bs[r][tx];
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] += as[r][ty + 8 * k] * bv;
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int i = ta * kG + ty + 8 * k, j = tb * kG + tx;
    if (i < a && j < b) partial[((int64_t)i * b + j) * gridDim.x + blockIdx.x] = acc[k];
  }
}

// out[e] = sum over chunks, in chunk order.
__global__ void gram_reduce(const double* __restrict__ partial, int nchunks, int64_t count,
                            double* __restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  double s = 0.0;
  for (int c = 0; c < nchunks; ++c) s += partial[e * nchunks + c];
  out[e] = s;
}

__global__ void combo_kernel(const double* __restrict__ V, int m, const double* __restrict__ G,
                             int q, double* __restrict__ Y, int add, int64_t n, int64_t ld) {
  extern __shared__ double g[];  // m x 8 slice of G
  const int c0 = blockIdx.y * 8;
  for (int t = threadIdx.x; t < m * 8; t += blockDim.x) {
    const int j = t >> 3, c = t & 7;
    g[t] = (c0 + c < q) ? G[(int64_t)j * q + c0 + c] : 0.0;
  }
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) acc[c] = (add && c0 + c < q) ? Y[(int64_t)(c0 + c) * ld + i] : 0.0;
  for (int j = 0; j < m; ++j) {
    const double v = V[(int64_t)j * ld + i];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] += v * g[j * 8 + c];
  }
#pragma unroll
  for (int c = 0; c < 8; ++c)
    if (c0 + c < q) Y[(int64_t)(c0 + c) * ld + i] = acc[c];
}

// out may be kv (each element is read before it is written by the same thread)
__global__ void sigma_image_kernel(const double* v, const double* kv,
                                   const double* __restrict__ wmax, double tau0, double tau1,
                                   double* out, int64_t n, int64_t ld) {
  const int64_t c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[c * ld + i] = tau0 * v[c * ld + i] / wmax[i] + tau1 * kv[c * ld + i];
}

__global__ void sub_cols_kernel(const double* __restrict__ a, const double* __restrict__ b,
                                double* __restrict__ out, int64_t n, int64_t ld) {
  const int64_t c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[c * ld + i] = a[c * ld + i] - b[c * ld + i];
}

// scales: sx[q], sb[q], sk0, sk1
__global__ void learn_features_kernel(const double* __restrict__ x, const double* __restrict__ b,
                                      const double* __restrict__ bnext,
                                      const double* __restrict__ w,
                                      const double* __restrict__ wnext,
                                      const double* __restrict__ diagk,
                                      const double* __restrict__ ku, int n_sk,
                                      const double* __restrict__ scales, double tau0, double tau1,
                                      double dmean, int64_t n, int64_t ld, int q,
                                      float* __restrict__ F) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t e = (int64_t)c * n + i, a = (int64_t)c * ld + i;
  const double sx = scales[c], sb = scales[q + c];
  const double wi = w[i] > 1e-30 ? w[i] : 1e-30, wn = wnext[i] > 1e-30 ? wnext[i] : 1e-30;
  const double d = 1.0 / (tau0 / wi + tau1);
  float f[16];
  f[0] = (float)(sx > 0.0 ? x[a] / sx : 0.0);
  f[1] = (float)(sb > 0.0 ? b[a] / sb : 0.0);
  f[2] = (float)(sb > 0.0 ? (bnext[a] - b[a]) / sb : 0.0);
  f[3] = (float)log(wn / wi);
  f[4] = (float)(d / dmean - 1.0);
  f[5] = (float)(diagk[i] - 1.0);
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const double sk = scales[2 * q + s];
    f[6 + s] = (float)(s < n_sk && sk > 0.0 ? ku[(int64_t)s * ld + i] / sk : 0.0);
  }
  f[14] = (float)tau1;
  f[15] = 0.f;
  float4* dst = reinterpret_cast<float4*>(F + e * 16);
#pragma unroll
  for (int k = 0; k < 4; ++k) dst[k] = make_float4(f[4 * k], f[4 * k + 1], f[4 * k + 2], f[4 * k + 3]);
}

__global__ void learn_targets_kernel(const double* __restrict__ x1, const double* __restrict__ x0,
                                     const double* __restrict__ s, int64_t n, int64_t ld,
                                     float* __restrict__ T) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t a = (int64_t)c * ld + i;
  T[(int64_t)c * n + i] = (float)(s[c] > 0.0 ? (x1[a] - x0[a]) / s[c] : 0.0);
}

__global__ void learn_to_cols_kernel(const float* __restrict__ y, int64_t n, int64_t ld,
                                     double* __restrict__ out) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[(int64_t)c * ld + i] = (double)y[(int64_t)c * n + i];
}

// Sample i per thread: sum over markers of z^2 (codes 00 -> 2, 10 -> 1, 11 -> 0,
// 01 missing -> 0), in the device word layout of the packed rows.
__global__ void grm_diag_kernel(const uint32_t* __restrict__ geno, int64_t wpr,
                                const double* __restrict__ two_p, const double* __restrict__ inv_s,
                                const uint8_t* __restrict__ excl, int64_t m, int64_t n,
                                double scale, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int e = (int)(i & 15), j = e >> 2, k = e & 3;
  const int shift = 16 * (j >> 1) + 2 * (j & 1) + 4 * k;
  const uint32_t* col = geno + (i >> 4);
  double s = 0.0;
  for (int64_t mk = 0; mk < m; ++mk) {
    if (excl && excl[mk]) continue;
    const uint32_t code = (__ldg(col + mk * wpr) >> shift) & 3u;
    if (code == 1u) continue;
    const double g = code == 0u ? 2.0 : (code == 2u ? 1.0 : 0.0);
    const double z = (g - __ldg(two_p + mk)) * __ldg(inv_s + mk);
    s += z * z;
  }
  out[i] = s * scale;
}

}  // namespace

size_t gram_partial_doubles(int64_t n, int a, int b) {
  return (size_t)gram_chunks(n, a, b) * (size_t)a * (size_t)b;
}

cudaError_t gram(const double* A, int a, const double* B, int b, int64_t n, int64_t ld,
                 double* partial, double* out, cudaStream_t st) {
  const int nch = gram_chunks(n, a, b);
  const int64_t chunk = round_up(ceil_div(n, nch), kG);
  const int tiles = ((a + kG - 1) / kG) * ((b + kG - 1) / kG);
  gram_kernel<<<dim3((unsigned)nch, (unsigned)tiles), kGThreads, 0, st>>>(A, a, B, b, n, ld, chunk,
                                                                           partial);
  const int64_t count = (int64_t)a * b;
  gram_reduce<<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(partial, nch, count, out);
  count_launches(2);
  return cudaGetLastError();
}

cudaError_t combo(const double* V, int m, const double* G, int q, double* Y, bool add, int64_t n,
                  int64_t ld, cudaStream_t st) {
  if (m <= 0 || q <= 0) return cudaSuccess;
  const dim3 grid((unsigned)ceil_div(n, 256), (unsigned)ceil_div(q, 8));
  combo_kernel<<<grid, 256, (size_t)m * 8 * sizeof(double), st>>>(V, m, G, q, Y, add ? 1 : 0, n,
                                                                  ld);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t sigma_image(const double* v, const double* kv, const double* wmax, double tau0,
                        double tau1, double* out, int64_t n, int64_t ld, int q, cudaStream_t st) {
  if (q <= 0) return cudaSuccess;
  sigma_image_kernel<<<dim3((unsigned)ceil_div(n, 256), (unsigned)q), 256, 0, st>>>(
      v, kv, wmax, tau0, tau1, out, n, ld);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t sub_cols(const double* a, const double* b, double* out, int64_t n, int64_t ld, int q,
                     cudaStream_t st) {
  if (q <= 0) return cudaSuccess;
  sub_cols_kernel<<<dim3((unsigned)ceil_div(n, 256), (unsigned)q), 256, 0, st>>>(a, b, out, n, ld);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t learn_features(const double* x, const double* b, const double* bnext, const double* w,
                           const double* wnext, const double* diagk, const double* ku, int n_sk,
                           const double* scales, double tau0, double tau1, double dmean,
                           int64_t n, int64_t ld, int q, float* F, cudaStream_t st) {
  learn_features_kernel<<<dim3((unsigned)ceil_div(n, 256), (unsigned)q), 256, 0, st>>>(
      x, b, bnext, w, wnext, diagk, ku, n_sk, scales, tau0, tau1, dmean, n, ld, q, F);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t learn_targets(const double* x1, const double* x0, const double* s, int64_t n,
                          int64_t ld, int q, float* T, cudaStream_t st) {
  learn_targets_kernel<<<dim3((unsigned)ceil_div(n, 256), (unsigned)q), 256, 0, st>>>(x1, x0, s, n,
                                                                                     ld, T);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t learn_to_cols(const float* y, int64_t n, int64_t ld, int q, double* out,
                          cudaStream_t st) {
  learn_to_cols_kernel<<<dim3((unsigned)ceil_div(n, 256), (unsigned)q), 256, 0, st>>>(y, n, ld, out);
  count_launches(1);
  return cudaGetLastError();
}

Status grm_diag(saige_grm* h, double* out, cudaStream_t st) {
  const int64_t m_used = h->masked ? h->m_active : h->m_eff;
  const double scale = m_used > 0 ? 1.0 / (double)m_used : 0.0;
  grm_diag_kernel<<<(unsigned)ceil_div(h->n, 256), 256, 0, st>>>(
      h->geno, h->wpr, h->two_p, h->inv_s, h->masked ? h->excl.as<uint8_t>() : nullptr, h->m, h->n,
      scale, out);
  count_launches(1);
  SG_CHECK_LAUNCH();
  return Status();
}

}  // namespace saige
