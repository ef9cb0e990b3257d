// Variance ratio of fit-null on the GPU: estimate_variance_ratio
// (saige-core/src/glmm/variance_ratio.rs:87-246) as fit_null.rs:290-373 drives it.
//
// The reference tries the candidate markers one at a time in a shuffled order,
// solving Sigma x = g_tilde for each with a single-vector PCG, until the
// coefficient of variation of the per-marker ratios is small enough.  Here the
// candidates are taken in the same order but in blocks: one block PCG (the
// GRM product costs nearly the same for 1 or 64 right-hand sides) solves a
// whole block, and the host then applies the reference's skip and stopping
// rules marker by marker, so the ratios used, their order and the stopping
// point are the reference's.  Each column's PCG recurrence is independent of
// the other columns of its block.
//
// X adjustment.  fit_null.rs:294-306 fills (X'WX)^-1 X'W as a p x n row-major
// array and reads it back with DenseMatrix::from_col_major(p, n, ..), so the
// matrix that multiplies g0 in variance_ratio.rs:145 has element (r, c) =
// data[c*p + r], not the projection coefficient (r, c).  SAIGE_VR_XADJUST_REFERENCE
// reproduces that array exactly; SAIGE_VR_XADJUST_PROJECTION applies the
// projection X (X'WX)^-1 X'W g.
//
// Missing calls.  The reference keeps them as NaN in the VR dosages (plink.rs:
// 170-179, fit_null.rs:248-253), which makes every affected ratio NaN.  Here a
// missing call is set to 2*af of the called genotypes of its marker before the
// allele flip, which leaves every marker without missing calls as in the
// reference.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <functional>
#include <vector>

#include "engine.cuh"
#include "kernels_vec.cuh"
#include "rng.hpp"
#include "vr.cuh"

namespace saige {
namespace {

constexpr int kT = 256;
constexpr int kMaxP = 64;

// stats[2c] = sum of the called dosages of column c, stats[2c+1] = their count.
// Both are integers below 2^53, so the atomic additions are exact in any order.
__global__ void vr_stats_kernel(const double* __restrict__ g, int64_t n, int64_t ld,
                                double* __restrict__ stats) {
  const int c = blockIdx.y;
  double s = 0.0, k = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = g[(int64_t)c * ld + i];
    if (!isnan(v)) {
      s += v;
      k += 1.0;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    k += __shfl_xor_sync(0xffffffffu, k, o);
  }
  __shared__ double ss[kT / 32], sk[kT / 32];
  if ((threadIdx.x & 31) == 0) {
    ss[threadIdx.x >> 5] = s;
    sk[threadIdx.x >> 5] = k;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < kT / 32; ++w) {
      a += ss[w];
      b += sk[w];
    }
    atomicAdd(&stats[2 * c], a);
    atomicAdd(&stats[2 * c + 1], b);
  }
}

// g = missing ? fill : g, then 2 - g when flipped; padding rows zero.
__global__ void vr_prep_kernel(double* __restrict__ g, int64_t n, int64_t ld,
                               const double* __restrict__ fill, const int32_t* __restrict__ flip) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ld) return;
  double v = 0.0;
  if (i < n) {
    v = g[(int64_t)c * ld + i];
    if (isnan(v)) v = fill[c];
    if (flip[c]) v = 2.0 - v;
  }
  g[(int64_t)c * ld + i] = v;
}

// A (n x p, column-major, ld) such that A' g0 is the vector the reference
// subtracts from (variance_ratio.rs:145).  With D[j*n + i] = sum_k inv(j,k)
// x(i,k) w(i) (fit_null.rs:297-303): scrambled, A(i, r) = D[i*p + r]; projection,
// A(i, r) = D[r*n + i].
__global__ void vr_adjust_matrix_kernel(const double* __restrict__ x, const double* __restrict__ w,
                                        const double* __restrict__ inv, int p, int64_t n,
                                        int64_t ld, int scrambled, double* __restrict__ a) {
  const int r = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ld) return;
  double val = 0.0;
  if (i < n) {
    const int64_t flat = scrambled ? i * p + r : (int64_t)r * n + i;
    const int64_t j = flat / n, ii = flat - j * n;
    for (int k = 0; k < p; ++k) val += inv[j * p + k] * x[(int64_t)k * ld + ii] * w[ii];
  }
  a[(int64_t)r * ld + i] = val;
}

// out[:, c] = s * g[:, c]
__global__ void vr_mul_rows_kernel(const double* __restrict__ s, const double* __restrict__ g,
                                   int64_t ld, double* __restrict__ out) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ld) out[(int64_t)c * ld + i] = s[i] * g[(int64_t)c * ld + i];
}

// Dosages of candidate markers from packed .bed rows in device memory (codes
// 00,01,10,11 -> 2, NaN, 1, 0 as plink.rs:170-179), samples in subset order.
__global__ void vr_bed_decode_kernel(const uint8_t* __restrict__ rows, int64_t bpm,
                                     const int64_t* __restrict__ markers,
                                     const int64_t* __restrict__ sample_idx, int64_t n, int64_t ld,
                                     double* __restrict__ out) {
  const int c = blockIdx.y;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t s = sample_idx ? sample_idx[i] : i;
  const uint8_t byte = rows[markers[c] * bpm + s / 4];
  const int code = (byte >> (2 * (s % 4))) & 3;
  out[(int64_t)c * ld + i] = code == 0 ? 2.0 : (code == 2 ? 1.0 : (code == 3 ? 0.0 : (double)NAN));
}

inline unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + kT - 1) / kT); }

// variance_ratio.rs:260-272: (sd / mean) / n, infinity for n <= 1 or |mean| < 1e-30.
double cal_cv(const std::vector<double>& v) {
  const size_t n = v.size();
  if (n <= 1) return INFINITY;
  double m = 0.0;
  for (double x : v) m += x;
  m /= (double)n;
  if (fabs(m) < 1e-30) return INFINITY;
  double var = 0.0;
  for (double x : v) var += (x - m) * (x - m);
  var /= ((double)n - 1.0);
  return (sqrt(var) / m) / (double)n;
}

bool cholesky_small(const double* a, int p, double* l) {
  for (int i = 0; i < p * p; ++i) l[i] = 0.0;
  for (int j = 0; j < p; ++j) {
    double sum = 0.0;
    for (int k = 0; k < j; ++k) sum += l[j * p + k] * l[j * p + k];
    const double diag = a[j * p + j] - sum;
    if (diag <= 0.0) return false;
    l[j * p + j] = sqrt(diag);
    for (int i = j + 1; i < p; ++i) {
      double s = 0.0;
      for (int k = 0; k < j; ++k) s += l[i * p + k] * l[j * p + k];
      l[i * p + j] = (a[i * p + j] - s) / l[j * p + j];
    }
  }
  return true;
}

void chol_solve_small(const double* l, int p, const double* b, double* x) {
  double y[kMaxP];
  for (int i = 0; i < p; ++i) {
    double s = 0.0;
    for (int j = 0; j < i; ++j) s += l[i * p + j] * y[j];
    y[i] = (b[i] - s) / l[i * p + i];
  }
  for (int i = p - 1; i >= 0; --i) {
    double s = 0.0;
    for (int j = i + 1; j < p; ++j) s += l[j * p + i] * x[j];
    x[i] = (y[i] - s) / l[i * p + i];
  }
}

}  // namespace

// Writes the raw dosages (NaN = missing) of candidates cand[0..B) into the
// columns of g (ld = n_pad, rows 0..n-1) on stream st.
using VrFill = std::function<Status(const std::vector<int64_t>& cand, double* g, cudaStream_t st)>;

Status vr_run(saige_grm* h, const VrFill& fill, int64_t n_cand, const double* mac, const double* mu,
              const double* w, const double tau[2], int trait, const double* x, int p,
              const saige_vr_config* cfg, saige_vr_summary* out, double* per_marker_vr,
              int64_t* used_idx) {
  const int64_t n = h->n, ld = h->n_pad;
  cudaStream_t st = h->stream;
  if (p <= 0 || p > kMaxP) return fail(SAIGE_EINVAL, "p must be in 1..%d", kMaxP);
  if (cfg->xadjust != SAIGE_VR_XADJUST_REFERENCE && cfg->xadjust != SAIGE_VR_XADJUST_PROJECTION)
    return fail(SAIGE_EINVAL, "unknown xadjust mode %d", cfg->xadjust);
  if (cfg->n_markers <= 0) return fail(SAIGE_EINVAL, "n_markers must be positive");
  *out = saige_vr_summary{};
  const int block = cfg->block > 0 ? std::min(cfg->block, 256)
                                   : (cfg->precision == SAIGE_PREC_MIXED ? 64 : 0);
  const int bmax = std::max(block, std::max(cfg->n_markers, 10));

  // device workspace: X, w, wmax, d, trait weights, A (n x p), G, x, tmp (n x bmax)
  DevBuf mem;
  const size_t vec_cols = (size_t)(2 * p + 4) + 3 * (size_t)bmax;
  const int nb = red_blocks(n);
  const size_t pw = (size_t)std::max(p, bmax);
  const size_t part = (size_t)nb * (size_t)p * pw;
  const size_t small = (size_t)p * p + 4 * (size_t)bmax + (size_t)p * pw + 2 * (size_t)bmax + 64;
  SG_TRY(mem.reserve((vec_cols * ld + part + small) * sizeof(double)));
  double* b = mem.as<double>();
  double* dX = b;        b += (size_t)p * ld;
  double* dA = b;        b += (size_t)p * ld;
  double* dw = b;        b += ld;
  double* dwmax = b;     b += ld;
  double* dd = b;        b += ld;
  double* dcw = b;       b += ld;
  double* dG = b;        b += (size_t)bmax * ld;
  double* dSol = b;      b += (size_t)bmax * ld;
  double* dTmp = b;      b += (size_t)bmax * ld;
  double* dPart = b;     b += part;
  double* dInv = b;      b += (size_t)p * p;
  double* dStats = b;    b += 2 * (size_t)bmax;
  double* dFill = b;     b += (size_t)bmax;
  int32_t* dFlip = reinterpret_cast<int32_t*>(b);  b += (size_t)bmax;
  double* dT = b;        // p x max(p, bmax), then 2 x bmax dots

  cudaEvent_t e0, e1;
  SG_CUDA(cudaEventCreate(&e0));
  SG_CUDA(cudaEventCreate(&e1));
  SG_CUDA(cudaEventRecord(e0, st));
  const int64_t kv0 = h->n_kv;

  // inputs (the padding rows of every column stay zero)
  SG_CUDA(cudaMemsetAsync(mem.ptr, 0, vec_cols * ld * sizeof(double), st));
  SG_CUDA(cudaMemcpy2DAsync(dX, (size_t)ld * 8, x, (size_t)n * 8, (size_t)n * 8, (size_t)p,
                            cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemcpyAsync(dw, w, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  {
    // variance_ratio.rs:162-180: mu(1-mu) for binary, mu for survival, 1 otherwise
    std::vector<double> cw((size_t)n);
    for (int64_t i = 0; i < n; ++i)
      cw[(size_t)i] = trait == SAIGE_TRAIT_BINARY ? mu[i] * (1.0 - mu[i])
                      : (trait == SAIGE_TRAIT_SURVIVAL ? mu[i] : 1.0);
    SG_CUDA(cudaMemcpyAsync(dcw, cw.data(), (size_t)n * 8, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaStreamSynchronize(st));
  }
  SG_CUDA(sigma_diag(dw, tau[0], tau[1], dwmax, dd, n, st));

  // fit_null.rs:291-293: XVX = X'WX, its inverse by unit-column Cholesky solves
  std::vector<double> xvx((size_t)p * p), l((size_t)p * p), inv((size_t)p * p);
  SG_CUDA(cross_dots(dX, p, dX, p, dw, n, ld, dPart, dT, st));
  SG_CUDA(cudaMemcpyAsync(xvx.data(), dT, (size_t)p * p * 8, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (!cholesky_small(xvx.data(), p, l.data()))
    return fail(SAIGE_SINGULAR, "X'WX is not positive definite (variance ratio)");
  for (int j = 0; j < p; ++j) {
    double e[kMaxP] = {0}, col[kMaxP];
    e[j] = 1.0;
    chol_solve_small(l.data(), p, e, col);
    for (int k = 0; k < p; ++k) inv[(size_t)k * p + j] = col[k];
  }
  SG_CUDA(cudaMemcpyAsync(dInv, inv.data(), (size_t)p * p * 8, cudaMemcpyHostToDevice, st));
  vr_adjust_matrix_kernel<<<dim3(blocks_for(ld), (unsigned)p), kT, 0, st>>>(
      dX, dw, dInv, p, n, ld, cfg->xadjust == SAIGE_VR_XADJUST_REFERENCE ? 1 : 0, dA);
  SG_CHECK_LAUNCH();
  count_launches(1);

  // the order in which variance_ratio.rs:116-120 tries the candidates
  std::vector<int64_t> order((size_t)n_cand);
  for (int64_t i = 0; i < n_cand; ++i) order[(size_t)i] = i;
  ChaCha8 rng(cfg->seed);
  rng.shuffle(order.data(), order.size());

  std::vector<double> vrs;
  std::vector<int64_t> used;
  int target = cfg->n_markers;
  bool stop = false;
  size_t pos = 0;
  while (!stop && pos < order.size()) {
    // next block of candidates that pass the MAC rule (variance_ratio.rs:124-126)
    const size_t want = block > 0 ? (size_t)block
                                  : (vrs.empty() ? (size_t)cfg->n_markers : (size_t)10);
    std::vector<int64_t> cand;
    while (pos < order.size() && cand.size() < std::min(want, (size_t)bmax)) {
      const int64_t idx = order[pos++];
      if (mac[idx] >= cfg->min_mac) cand.push_back(idx);
    }
    if (cand.empty()) break;
    const int q = (int)cand.size();
    out->n_blocks += 1;
    out->n_solved += q;
    SG_TRY(fill(cand, dG, st));
    // per-candidate counts -> fill value, allele flip, AC (variance_ratio.rs:131-142)
    SG_CUDA(cudaMemsetAsync(dStats, 0, 2 * (size_t)q * 8, st));
    vr_stats_kernel<<<dim3((unsigned)std::min<int64_t>(blocks_for(n), 296), (unsigned)q), kT, 0,
                      st>>>(dG, n, ld, dStats);
    SG_CHECK_LAUNCH();
    std::vector<double> stats(2 * (size_t)q), fillv((size_t)q), ac((size_t)q);
    std::vector<int32_t> flip((size_t)q);
    SG_CUDA(cudaMemcpyAsync(stats.data(), dStats, 2 * (size_t)q * 8, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    for (int c = 0; c < q; ++c) {
      const double s_nm = stats[2 * (size_t)c], n_nm = stats[2 * (size_t)c + 1];
      fillv[(size_t)c] = n_nm > 0.0 ? 2.0 * (s_nm / (2.0 * n_nm)) : 0.0;
      const double sum = s_nm + ((double)n - n_nm) * fillv[(size_t)c];
      const double af = sum / (2.0 * (double)n);
      flip[(size_t)c] = af > 0.5 ? 1 : 0;
      ac[(size_t)c] = flip[(size_t)c] ? 2.0 * (double)n - sum : sum;
    }
    SG_CUDA(cudaMemcpyAsync(dFill, fillv.data(), (size_t)q * 8, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(dFlip, flip.data(), (size_t)q * 4, cudaMemcpyHostToDevice, st));
    vr_prep_kernel<<<dim3(blocks_for(ld), (unsigned)q), kT, 0, st>>>(dG, n, ld, dFill, dFlip);
    SG_CHECK_LAUNCH();
    // X adjustment: G -= X (A' G)
    SG_CUDA(cross_dots(dA, p, dG, q, nullptr, n, ld, dPart, dT, st));
    SG_CUDA(sub_combo(dG, q, dX, p, dT, n, ld, st));
    // Sigma^-1 g_tilde for the whole block (PcgSolver::new(1e-5, 500), zero start)
    PcgRun run;
    run.b = dG;
    run.x0 = nullptr;
    run.wv = dwmax;
    run.d = dd;
    run.tau0 = tau[0];
    run.tau1 = tau[1];
    run.q = q;
    run.tol = 1e-5;
    run.max_iter = 500;
    run.precision = cfg->precision;
    run.x = dSol;
    SG_TRY(pcg_run(h, run, st));
    out->pcg_iters += run.total_iters;
    // var1 * AC = g_tilde' Sigma^-1 g_tilde; var2 * AC = sum c g_tilde^2
    double* dDots = dT;
    SG_CUDA(col_dots(dG, dSol, n, ld, q, dPart, dDots, st));
    vr_mul_rows_kernel<<<dim3(blocks_for(ld), (unsigned)q), kT, 0, st>>>(dcw, dG, ld, dTmp);
    SG_CHECK_LAUNCH();
    SG_CUDA(col_dots(dTmp, dG, n, ld, q, dPart, dDots + q, st));
    count_launches(3);
    std::vector<double> dots(2 * (size_t)q);
    SG_CUDA(cudaMemcpyAsync(dots.data(), dDots, 2 * (size_t)q * 8, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    // the reference's rules, marker by marker in shuffled order (variance_ratio.rs:139-210)
    for (int c = 0; c < q && !stop; ++c) {
      if (ac[(size_t)c] < 1.0) continue;
      const double var1 = dots[(size_t)c] / ac[(size_t)c];
      const double var2 = dots[(size_t)q + c] / ac[(size_t)c];
      if (var2 < 1e-30) continue;
      vrs.push_back(var1 / var2);
      used.push_back(cand[(size_t)c]);
      if ((int)vrs.size() >= target) {
        if (cal_cv(vrs) <= cfg->ratio_cv_cutoff) stop = true;
        else target += 10;
      }
    }
  }
  SG_CUDA(cudaEventRecord(e1, st));
  SG_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  out->seconds = ms * 1e-3;
  out->n_kv = h->n_kv - kv0;
  out->n_markers_used = (int32_t)vrs.size();
  if (vrs.empty()) return fail(SAIGE_EINVAL, "No markers available for variance ratio estimation");
  double mean = 0.0;
  for (double v : vrs) mean += v;
  out->variance_ratio = mean / (double)vrs.size();
  if (per_marker_vr) std::copy(vrs.begin(), vrs.end(), per_marker_vr);
  if (used_idx) std::copy(used.begin(), used.end(), used_idx);
  if (cfg->use_categorical) {
    // variance_ratio.rs:276-298 with the default MAC bins
    static const double lo[8] = {0.5, 1.5, 2.5, 3.5, 4.5, 5.5, 10.5, 20.5};
    static const double hi[8] = {1.5, 2.5, 3.5, 4.5, 5.5, 10.5, 20.5, INFINITY};
    for (int k = 0; k < 8; ++k) {
      double s = 0.0;
      int cnt = 0;
      for (size_t i = 0; i < vrs.size(); ++i) {
        const double mc = mac[used[i]];
        if (mc > lo[k] && mc <= hi[k]) {
          s += vrs[i];
          ++cnt;
        }
      }
      if (cnt > 0) {
        out->cat_upper[out->n_categories] = hi[k];
        out->cat_vr[out->n_categories] = s / (double)cnt;
        ++out->n_categories;
      }
    }
  }
  return Status();
}

}  // namespace saige

namespace saige {

Status vr_gather_rows(const uint8_t* bed_dev, int64_t bpm, const int64_t* vidx, int64_t m_vr,
                      const int64_t* sample_idx, int64_t n, VrRows& out, cudaStream_t st) {
  out.bpm = bpm;
  out.m = m_vr;
  out.has_sidx = sample_idx != nullptr;
  if (m_vr > 0) {
    SG_TRY(out.rows.reserve((size_t)m_vr * (size_t)bpm));
    for (int64_t j = 0; j < m_vr; ++j)
      SG_CUDA(cudaMemcpyAsync(out.rows.as<uint8_t>() + j * bpm, bed_dev + 3 + vidx[j] * bpm,
                              (size_t)bpm, cudaMemcpyDeviceToDevice, st));
  }
  if (sample_idx) {
    SG_TRY(out.sidx.reserve((size_t)n * sizeof(int64_t)));
    SG_CUDA(cudaMemcpyAsync(out.sidx.ptr, sample_idx, (size_t)n * sizeof(int64_t),
                            cudaMemcpyHostToDevice, st));
  }
  SG_CUDA(cudaStreamSynchronize(st));
  return Status();
}

Status vr_from_rows(saige_grm* h, const VrRows& rows, const double* mac, const double* mu,
                    const double* w, const double tau[2], int trait, const double* x, int p,
                    const saige_vr_config* cfg, saige_vr_summary* out) {
  const int64_t n = h->n, ld = h->n_pad;
  DevBuf dmarkers;
  SG_TRY(dmarkers.reserve(256 * sizeof(int64_t)));
  VrFill fill = [&](const std::vector<int64_t>& cand, double* g, cudaStream_t st) -> Status {
    SG_CUDA(cudaMemcpyAsync(dmarkers.ptr, cand.data(), cand.size() * sizeof(int64_t),
                            cudaMemcpyHostToDevice, st));
    vr_bed_decode_kernel<<<dim3(blocks_for(n), (unsigned)cand.size()), kT, 0, st>>>(
        rows.rows.as<uint8_t>(), rows.bpm, dmarkers.as<int64_t>(),
        rows.has_sidx ? rows.sidx.as<int64_t>() : nullptr, n, ld, g);
    count_launches(1);
    SG_CUDA(cudaGetLastError());
    // the host vector of indices must outlive the copy
    SG_CUDA(cudaStreamSynchronize(st));
    return Status();
  };
  return vr_run(h, fill, rows.m, mac, mu, w, tau, trait, x, p, cfg, out, nullptr, nullptr);
}

}  // namespace saige

using namespace saige;

#define SG_API extern "C" __attribute__((visibility("default")))

SG_API int32_t saige_vr_config_default(saige_vr_config* c) {
  if (!c) return fail(SAIGE_EINVAL, "null argument").code;
  // VarianceRatioConfig::default (variance_ratio.rs:45-56)
  *c = saige_vr_config{};
  c->n_markers = 30;
  c->use_categorical = 0;
  c->min_mac = 20.0;
  c->ratio_cv_cutoff = 0.001;
  c->seed = 12345;
  c->precision = SAIGE_PREC_FP32;
  c->xadjust = SAIGE_VR_XADJUST_REFERENCE;
  c->block = 0;
  return SAIGE_OK;
}

SG_API int32_t saige_vr_marker_order(uint64_t seed, int64_t n_cand, int64_t* order) {
  try {
    set_error("");
    if (!order || n_cand < 0) return fail(SAIGE_EINVAL, "null argument or n_cand < 0").code;
    for (int64_t i = 0; i < n_cand; ++i) order[i] = i;
    ChaCha8 rng(seed);
    rng.shuffle(order, (size_t)n_cand);
    return SAIGE_OK;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}

SG_API int32_t saige_estimate_variance_ratio(saige_grm* h, const double* dosages, const double* mac,
                                             int64_t n_cand, const double* mu, const double* w,
                                             const double tau[2], int32_t trait, const double* x,
                                             int32_t p, const saige_vr_config* cfg,
                                             saige_vr_summary* out, double* per_marker_vr,
                                             int64_t* used_idx) {
  try {
    set_error("");
    if (!h || !dosages || !mac || !mu || !w || !tau || !x || !out)
      return fail(SAIGE_EINVAL, "null argument").code;
    if (n_cand < 0) return fail(SAIGE_EINVAL, "n_cand < 0").code;
    if (trait < 0 || trait > 2) return fail(SAIGE_EINVAL, "unknown trait type").code;
    saige_vr_config c;
    if (cfg) c = *cfg;
    else saige_vr_config_default(&c);
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    const int64_t n = h->n, ld = h->n_pad;
    VrFill fill = [dosages, n, ld](const std::vector<int64_t>& cand, double* g,
                                   cudaStream_t st) -> Status {
      for (size_t k = 0; k < cand.size(); ++k)
        SG_CUDA(cudaMemcpyAsync(g + (int64_t)k * ld, dosages + cand[k] * n, (size_t)n * 8,
                                cudaMemcpyHostToDevice, st));
      return Status();
    };
    Status s = vr_run(h, fill, n_cand, mac, mu, w, tau, trait, x, p, &c, out, per_marker_vr,
                      used_idx);
    if (prev >= 0) cudaSetDevice(prev);
    return s.code;
  } catch (const std::bad_alloc&) {
    return fail(SAIGE_ENOMEM, "host allocation failed").code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}
