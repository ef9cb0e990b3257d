// Synthetic cohort generation (test and benchmark input; no counterpart in
// the reference).  The device kernel and the threaded host loop evaluate the
// same counter-based hash functions, so they write identical bytes.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "cohort.cuh"
#include "common.cuh"

using namespace saige;
using namespace saige::cohort;

namespace {

__global__ void gen_bed_kernel(Layout L, uint8_t* __restrict__ bed, int64_t bpm) {
  const int64_t total = L.m * bpm;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = t / bpm, b = t - m * bpm;
    const double p = allele_freq(L, m);
    bed[3 + t] = bed_byte(L, m, b, p);
  }
}

unsigned host_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t == 0 ? 1 : std::min(t, 64u);
}

template <class F>
void parallel_for(int64_t n, F f) {
  const unsigned nt = host_threads();
  std::vector<std::thread> th;
  const int64_t chunk = (n + nt - 1) / nt;
  for (unsigned k = 0; k < nt; ++k) {
    const int64_t lo = k * chunk, hi = std::min<int64_t>(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([=]() { f(lo, hi); });
  }
  for (auto& t : th) t.join();
}

double normal(uint64_t h1, uint64_t h2) {
  // Box-Muller on two hash uniforms (u1 in (0,1])
  const double u1 = 1.0 - u01(h1);
  const double u2 = u01(h2);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

Status check_spec(const saige_cohort_spec* s) {
  if (!s) return fail(SAIGE_EINVAL, "null spec");
  if (s->n <= 0 || s->m <= 0) return fail(SAIGE_EINVAL, "n and m must be positive");
  if (!(s->maf_lo > 0.0 && s->maf_lo <= s->maf_hi && s->maf_hi <= 0.5))
    return fail(SAIGE_EINVAL, "need 0 < maf_lo <= maf_hi <= 0.5");
  if (s->missing_rate < 0.0 || s->missing_rate >= 1.0)
    return fail(SAIGE_EINVAL, "missing_rate must be in [0, 1)");
  if (s->n_covar < 0 || s->n_covar > 63) return fail(SAIGE_EINVAL, "n_covar must be in 0..63");
  return Status();
}

}  // namespace

#define SG_API extern "C" __attribute__((visibility("default")))

SG_API int32_t saige_gen_bed(const saige_cohort_spec* spec, uint8_t* bed_out, int32_t on_device) {
  set_error("");
  Status s = check_spec(spec);
  if (!s.ok()) return s.code;
  if (!bed_out) return fail(SAIGE_EINVAL, "null output").code;
  const Layout L = make_layout(*spec);
  const int64_t bpm = (spec->n + 3) / 4;
  const uint8_t hdr[3] = {0x6C, 0x1B, 0x01};
  if (on_device) {
    if (cudaMemcpy(bed_out, hdr, 3, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(SAIGE_ECUDA, "header copy failed: %s", cudaGetErrorString(cudaGetLastError())).code;
    gen_bed_kernel<<<148 * 16, 256>>>(L, bed_out, bpm);
    count_launches(1);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(SAIGE_ECUDA, "gen_bed_kernel: %s", cudaGetErrorString(e)).code;
    return SAIGE_OK;
  }
  memcpy(bed_out, hdr, 3);
  parallel_for(spec->m, [&](int64_t lo, int64_t hi) {
    for (int64_t m = lo; m < hi; ++m) {
      const double p = allele_freq(L, m);
      uint8_t* row = bed_out + 3 + m * bpm;
      for (int64_t b = 0; b < bpm; ++b) row[b] = bed_byte(L, m, b, p);
    }
  });
  return SAIGE_OK;
}

SG_API int32_t saige_gen_pheno(const saige_cohort_spec* spec, double* y, double* x) {
  set_error("");
  Status s = check_spec(spec);
  if (!s.ok()) return s.code;
  if (!y || !x) return fail(SAIGE_EINVAL, "null output").code;
  const Layout L = make_layout(*spec);
  const int64_t n = spec->n;
  const int p = 1 + spec->n_covar;
  // covariates: intercept, N(0,1), Bernoulli(0.5), then N(0,1)
  std::vector<double> beta((size_t)p, 0.0);
  for (int64_t i = 0; i < n; ++i) x[i] = 1.0;
  for (int k = 1; k < p; ++k) {
    beta[(size_t)k] = k == 1 ? 0.3 : (k == 2 ? 0.2 : 0.1);
    for (int64_t i = 0; i < n; ++i) {
      double v;
      if (k == 2) v = u01(hash4(L.seed, kTagCov, (uint64_t)i, (uint64_t)(2 * k))) < 0.5 ? 1.0 : 0.0;
      else v = normal(hash4(L.seed, kTagCov, (uint64_t)i, (uint64_t)(2 * k)),
                      hash4(L.seed, kTagCov, (uint64_t)i, (uint64_t)(2 * k + 1)));
      x[(int64_t)k * n + i] = v;
    }
  }
  // polygenic score over evenly spaced causal markers, true genotypes
  const int64_t nc = std::max<int64_t>(1, std::min<int64_t>(spec->n_causal > 0 ? spec->n_causal : 500,
                                                           spec->m));
  const int64_t stride = spec->m / nc;
  std::vector<double> pgs((size_t)n, 0.0);
  parallel_for(n, [&](int64_t lo, int64_t hi) {
    for (int64_t c = 0; c < nc; ++c) {
      const int64_t m = c * stride;
      const double pm = allele_freq(L, m);
      const double sd = sqrt(2.0 * pm * (1.0 - pm));
      const double b = normal(hash4(L.seed, kTagEffect, (uint64_t)m, 0),
                              hash4(L.seed, kTagEffect, (uint64_t)m, 1));
      for (int64_t i = lo; i < hi; ++i)
        pgs[(size_t)i] += b * ((double)true_genotype(L, m, i, pm) - 2.0 * pm) / sd;
    }
  });
  double mean = 0.0, var = 0.0;
  for (double v : pgs) mean += v;
  mean /= (double)n;
  for (double v : pgs) var += (v - mean) * (v - mean);
  var /= (double)n;
  const double sdv = var > 0 ? sqrt(var) : 1.0;
  for (auto& v : pgs) v = (v - mean) / sdv;
  std::vector<double> lin((size_t)n, 0.0);
  for (int64_t i = 0; i < n; ++i) {
    double e = 0.0;
    for (int k = 1; k < p; ++k) e += beta[(size_t)k] * x[(int64_t)k * n + i];
    lin[(size_t)i] = e;
  }
  if (spec->trait == SAIGE_TRAIT_QUANTITATIVE) {
    const double h2 = spec->h2;
    for (int64_t i = 0; i < n; ++i) {
      const double eps = normal(hash4(L.seed, kTagNoise, (uint64_t)i, 0),
                                hash4(L.seed, kTagNoise, (uint64_t)i, 1));
      y[i] = lin[(size_t)i] + sqrt(h2) * pgs[(size_t)i] + sqrt(1.0 - h2) * eps;
    }
    return SAIGE_OK;
  }
  // binary: liability-scale genetic sd for h2 on the logistic scale,
  // intercept by bisection so that the mean risk equals the prevalence
  const double h2 = spec->h2 < 0.99 ? spec->h2 : 0.99;
  const double sg = sqrt(h2 * (M_PI * M_PI / 3.0) / (1.0 - h2));
  const double prev = spec->prevalence > 0 && spec->prevalence < 1 ? spec->prevalence : 0.1;
  double lo = -30.0, hi = 30.0;
  for (int it = 0; it < 100; ++it) {
    const double mid = 0.5 * (lo + hi);
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += 1.0 / (1.0 + exp(-(mid + lin[(size_t)i] + sg * pgs[(size_t)i])));
    if (s / (double)n < prev) lo = mid;
    else hi = mid;
  }
  const double b0 = 0.5 * (lo + hi);
  for (int64_t i = 0; i < n; ++i) {
    const double mu = 1.0 / (1.0 + exp(-(b0 + lin[(size_t)i] + sg * pgs[(size_t)i])));
    y[i] = u01(hash4(L.seed, kTagY, (uint64_t)i, 0)) < mu ? 1.0 : 0.0;
  }
  return SAIGE_OK;
}
