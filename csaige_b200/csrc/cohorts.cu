// Fit-null of several sub-cohorts of one .bed (different sample subsets, the same
// markers), as fit_null::run would do for each (saige-cli/src/commands/fit_null.rs:
// 199-287: counts, QC and the VR/GRM split over the cohort's samples, the GRM, the
// AI-REML fit).  The .bed is uploaded once.  Run concurrently, each cohort's fit owns
// a handle with its own stream on its own host thread, so that the launches of small
// cohorts — whose sample-side pass fills a fraction of the GPU and whose PCG steps
// are latency-bound — overlap with those of the others.
#include <stdint.h>
#include <string.h>

#include <chrono>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

using namespace saige;

#define SG_API extern "C" __attribute__((visibility("default")))

namespace {

struct CohortJob {
  const int64_t* sidx;
  int64_t n;
  const double* y;
  const double* x;
  saige_ai_reml_summary* out;
  double* alpha;
  int64_t m_grm = 0;
  int32_t rc = SAIGE_OK;
  std::string err;
};

void run_cohort(int device, const uint8_t* d_bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                int32_t p, int32_t trait, double min_maf, double max_missing,
                const saige_ai_reml_config* cfg, CohortJob& job) {
  cudaSetDevice(device);
  std::vector<double> af((size_t)m_tot), mac((size_t)m_tot);
  std::vector<int64_t> nv((size_t)m_tot);
  int32_t rc = saige_bed_marker_stats_dev(d_bed, bed_len, n_fam, m_tot, job.sidx, job.n,
                                          af.data(), mac.data(), nv.data());
  std::vector<int64_t> gidx((size_t)m_tot), vidx((size_t)m_tot);
  int64_t m_grm = 0, m_vr = 0;
  if (rc == SAIGE_OK)
    rc = saige_select_grm_markers(af.data(), mac.data(), nv.data(), m_tot, job.n, min_maf,
                                  max_missing, cfg->seed, gidx.data(), &m_grm, vidx.data(), &m_vr);
  saige_grm* h = nullptr;
  if (rc == SAIGE_OK) {
    std::vector<double> gaf((size_t)m_grm);
    for (int64_t j = 0; j < m_grm; ++j) gaf[(size_t)j] = af[(size_t)gidx[(size_t)j]];
    rc = saige_grm_create_from_bed_dev(d_bed, bed_len, n_fam, m_tot, job.sidx, job.n, gidx.data(),
                                       m_grm, gaf.data(), device, &h);
  }
  if (rc == SAIGE_OK)
    rc = saige_fit_ai_reml(h, job.y, job.x, job.n, p, trait, cfg, job.out, job.alpha, nullptr,
                           nullptr, nullptr, nullptr);
  if (rc != SAIGE_OK) job.err = saige_last_error();
  if (h) saige_grm_destroy(h);
  job.m_grm = m_grm;
  job.rc = rc;
}

}  // namespace

SG_API int32_t saige_fit_null_cohorts(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                      int64_t m_tot, int32_t n_cohorts,
                                      const int64_t* const* sample_idx, const int64_t* n,
                                      const double* const* y, const double* const* x, int32_t p,
                                      int32_t trait, double min_maf, double max_missing,
                                      const saige_ai_reml_config* cfg, int32_t concurrent,
                                      saige_ai_reml_summary* out, double* const* alpha,
                                      int64_t* m_grm, double* wall_seconds) {
  try {
    set_error("");
    if (!bed || !sample_idx || !n || !y || !x || !out || n_cohorts <= 0 || m_tot <= 0)
      return fail(SAIGE_EINVAL, "null argument").code;
    for (int32_t c = 0; c < n_cohorts; ++c)
      if (!sample_idx[c] || n[c] <= 0 || !y[c] || !x[c])
        return fail(SAIGE_EINVAL, "cohort %d: null argument or empty", c).code;
    saige_ai_reml_config cf;
    if (cfg) cf = *cfg;
    else saige_ai_reml_config_default(&cf);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(SAIGE_ECUDA, "no CUDA device").code;
    const auto t0 = std::chrono::steady_clock::now();
    DevBuf d_bed;
    Status s = d_bed.reserve(bed_len);
    if (!s.ok()) return s.code;
    if (cudaMemcpy(d_bed.ptr, bed, bed_len, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(SAIGE_ECUDA, "bed upload failed: %s", cudaGetErrorString(cudaGetLastError())).code;
    std::vector<CohortJob> jobs((size_t)n_cohorts);
    for (int32_t c = 0; c < n_cohorts; ++c) {
      CohortJob& j = jobs[(size_t)c];
      j.sidx = sample_idx[c];
      j.n = n[c];
      j.y = y[c];
      j.x = x[c];
      j.out = out + c;
      j.alpha = alpha ? alpha[c] : nullptr;
    }
    const uint8_t* db = d_bed.as<uint8_t>();
    if (concurrent) {
      std::vector<std::thread> th;
      th.reserve((size_t)n_cohorts);
      for (int32_t c = 0; c < n_cohorts; ++c)
        th.emplace_back(run_cohort, dev, db, bed_len, n_fam, m_tot, p, trait, min_maf, max_missing,
                        &cf, std::ref(jobs[(size_t)c]));
      for (auto& t : th) t.join();
    } else {
      for (int32_t c = 0; c < n_cohorts; ++c)
        run_cohort(dev, db, bed_len, n_fam, m_tot, p, trait, min_maf, max_missing, &cf,
                   jobs[(size_t)c]);
    }
    d_bed.release();
    if (wall_seconds)
      *wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int32_t c = 0; c < n_cohorts; ++c) {
      if (m_grm) m_grm[c] = jobs[(size_t)c].m_grm;
      if (jobs[(size_t)c].rc != SAIGE_OK)
        return fail(jobs[(size_t)c].rc, "cohort %d: %s", c, jobs[(size_t)c].err.c_str()).code;
    }
    return SAIGE_OK;
  } catch (const std::bad_alloc&) {
    return fail(SAIGE_ENOMEM, "host allocation failed").code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}
