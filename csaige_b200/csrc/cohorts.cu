// Fit-null of several sub-cohorts of one .bed (different sample subsets, the same
// markers), as fit_null::run would do for each (saige-cli/src/commands/fit_null.rs:
// 199-287: counts, QC and the VR/GRM split over the cohort's samples, the GRM, the
// AI-REML fit).  The .bed is uploaded once.
//
// Sequential: each cohort in turn, every step its own (as fit_null::run per cohort).
// Concurrent: the .bed streams in by marker chunks, and one launch per chunk counts
// every cohort's alleles and missing calls of the chunk's markers (each raw row staged
// once for all cohorts), all under the PCIe-bound transfer.  For MIXED fits the host
// applies each cohort's marker QC to every chunk as its counts arrive and one more
// launch per chunk gathers the passing markers into every cohort's GRM, also under the
// transfer (stream_cohorts); FP32 fits select their markers once all counts are in and
// gather in one pass after the upload (build_handles).  The fits then run on a pool of
// host threads, each cohort on its own stream, so that the launches of small cohorts —
// whose sample-side pass fills a fraction of the GPU and whose PCG steps are
// latency-bound — overlap with those of the others.  Counts and rows are exact either
// way, so both orders give the same fits.
#include <stdint.h>
#include <string.h>

#include <math.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.cuh"
#include "kernels.cuh"

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
  // marker statistics over the cohort's samples, when counted beforehand
  bool have_stats = false;
  std::vector<double> af, mac;
  std::vector<int64_t> nv;
  // the cohort's GRM handle, when built beforehand (rows from the shared gather)
  saige_grm* h = nullptr;
  std::vector<int64_t> gidx;
  std::vector<double> gaf;
  int64_t m_grm = 0;
  int32_t rc = SAIGE_OK;
  std::string err;
};

void run_cohort(int device, const uint8_t* d_bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                int32_t p, int32_t trait, double min_maf, double max_missing,
                const saige_ai_reml_config* cfg, CohortJob& job) {
  cudaSetDevice(device);
  if (job.h) {  // handle built beforehand: only the fit
    int32_t rc = saige_fit_ai_reml(job.h, job.y, job.x, job.n, p, trait, cfg, job.out, job.alpha,
                                   nullptr, nullptr, nullptr, nullptr);
    if (rc != SAIGE_OK) job.err = saige_last_error();
    grm_shell_destroy(job.h);
    job.h = nullptr;
    job.rc = rc;
    return;
  }
  int32_t rc = SAIGE_OK;
  if (!job.have_stats) {
    job.af.resize((size_t)m_tot);
    job.mac.resize((size_t)m_tot);
    job.nv.resize((size_t)m_tot);
    rc = saige_bed_marker_stats_dev(d_bed, bed_len, n_fam, m_tot, job.sidx, job.n, job.af.data(),
                                    job.mac.data(), job.nv.data());
  }
  std::vector<int64_t> gidx((size_t)m_tot), vidx((size_t)m_tot);
  int64_t m_grm = 0, m_vr = 0;
  if (rc == SAIGE_OK)
    rc = saige_select_grm_markers(job.af.data(), job.mac.data(), job.nv.data(), m_tot, job.n,
                                  min_maf, max_missing, cfg->seed, gidx.data(), &m_grm,
                                  vidx.data(), &m_vr);
  saige_grm* h = nullptr;
  if (rc == SAIGE_OK) {
    std::vector<double> gaf((size_t)m_grm);
    for (int64_t j = 0; j < m_grm; ++j) gaf[(size_t)j] = job.af[(size_t)gidx[(size_t)j]];
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

// Every cohort's sample indices on the device, each list padded to 16 entries.
struct SampleLists {
  DevBuf d_sidx;
  std::vector<int64_t> offs;
};

// Uploads the .bed into d_bed in marker chunks on a copy stream while, chunk by chunk,
// one launch counts every cohort's alleles and missing calls of the chunk's markers;
// fills each job's marker statistics and leaves the sample lists on the device.
Status upload_and_count(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                        DevBuf& d_bed, std::vector<CohortJob>& jobs, SampleLists& lists) {
  const int64_t bpm = (n_fam + 3) / 4;
  const int k = (int)jobs.size();
  // every cohort's sample list, each padded to a multiple of 16 entries
  std::vector<int32_t> all;
  std::vector<int64_t> offs((size_t)k), ns((size_t)k);
  for (int c = 0; c < k; ++c) {
    std::vector<int32_t> s;
    bool identity = true;
    SG_TRY(check_subset(jobs[(size_t)c].sidx, jobs[(size_t)c].n, n_fam, s, identity));
    offs[(size_t)c] = (int64_t)all.size();
    ns[(size_t)c] = jobs[(size_t)c].n;
    if (jobs[(size_t)c].sidx) {
      all.insert(all.end(), s.begin(), s.end());
    } else {
      for (int64_t i = 0; i < n_fam; ++i) all.push_back((int32_t)i);
    }
    all.resize((size_t)round_up((int64_t)all.size(), 16), 0);
  }
  cudaStream_t cp = nullptr, kst = nullptr;
  std::vector<cudaEvent_t> ev;
  DevBuf& d_sidx = lists.d_sidx;
  lists.offs = offs;
  DevBuf d_offs, d_ns, d_cnt;
  std::vector<long long> cnt;
  auto body = [&]() -> Status {
    SG_CUDA(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking));
    SG_CUDA(cudaStreamCreateWithFlags(&kst, cudaStreamNonBlocking));
    SG_TRY(d_sidx.reserve(all.size() * 4));
    SG_TRY(d_offs.reserve((size_t)k * 8));
    SG_TRY(d_ns.reserve((size_t)k * 8));
    SG_TRY(d_cnt.reserve((size_t)k * m_tot * 16));
    SG_CUDA(cudaMemcpyAsync(d_sidx.ptr, all.data(), all.size() * 4, cudaMemcpyHostToDevice, kst));
    SG_CUDA(cudaMemcpyAsync(d_offs.ptr, offs.data(), (size_t)k * 8, cudaMemcpyHostToDevice, kst));
    SG_CUDA(cudaMemcpyAsync(d_ns.ptr, ns.data(), (size_t)k * 8, cudaMemcpyHostToDevice, kst));
    // every chunk's copy is queued first; the counts follow chunk by chunk
    constexpr int kChunks = 32;
    const int64_t per = std::max<int64_t>(1, ceil_div(m_tot, (int64_t)kChunks));
    uint8_t* dst = d_bed.as<uint8_t>();
    std::vector<std::pair<int64_t, int64_t>> spans;
    for (int64_t j0 = 0; j0 < m_tot; j0 += per) {
      const int64_t j1 = std::min(m_tot, j0 + per);
      const size_t lo = j0 == 0 ? 0 : (size_t)(3 + j0 * bpm);
      const size_t hi = j1 == m_tot ? bed_len : (size_t)(3 + j1 * bpm);
      SG_CUDA(cudaMemcpyAsync(dst + lo, bed + lo, hi - lo, cudaMemcpyHostToDevice, cp));
      cudaEvent_t e = nullptr;
      SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev.push_back(e);
      SG_CUDA(cudaEventRecord(e, cp));
      spans.emplace_back(j0, j1);
    }
    for (size_t i = 0; i < spans.size(); ++i) {
      SG_CUDA(cudaStreamWaitEvent(kst, ev[i], 0));
      SG_CUDA(launch_bed_count_cohorts(dst, bpm, spans[i].first, spans[i].second - spans[i].first,
                                       d_sidx.as<int32_t>(), d_offs.as<int64_t>(),
                                       d_ns.as<int64_t>(), k, m_tot, d_cnt.as<long long>(), kst));
    }
    cnt.resize((size_t)k * m_tot * 2);
    SG_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt.ptr, cnt.size() * 8, cudaMemcpyDeviceToHost, kst));
    SG_CUDA(cudaStreamSynchronize(kst));
    SG_CUDA(cudaStreamSynchronize(cp));
    return Status();
  };
  Status s = body();
  if (cp) cudaStreamSynchronize(cp);
  if (kst) cudaStreamSynchronize(kst);
  {
    ReleaseScope idle(ReleaseMode::kIdle, nullptr);  // both streams have drained
    d_offs.release();
    d_ns.release();
    d_cnt.release();
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  if (cp) cudaStreamDestroy(cp);
  if (kst) cudaStreamDestroy(kst);
  SG_TRY(s);
  for (int c = 0; c < k; ++c) {
    CohortJob& j = jobs[(size_t)c];
    j.af.resize((size_t)m_tot);
    j.mac.resize((size_t)m_tot);
    j.nv.resize((size_t)m_tot);
    stats_from_counts(cnt.data() + (size_t)c * m_tot * 2, m_tot, j.n, j.af.data(), j.mac.data(),
                      j.nv.data());
    j.have_stats = true;
  }
  return Status();
}

// Host-mapped memory for the counts and row maps of a streamed cohort build (read and
// written by kernels over PCIe: no copy queues behind the .bed's chunks on the copy
// engine).  One block is kept for the process; a call that finds it in use by another
// thread takes a block of its own.
std::mutex g_cmap_mu;
void* g_cmap = nullptr;
size_t g_cmap_bytes = 0;
bool g_cmap_busy = false;

}  // namespace

void saige::release_cohort_mapped() {
  std::lock_guard<std::mutex> lk(g_cmap_mu);
  if (g_cmap && !g_cmap_busy) {
    cudaFreeHost(g_cmap);
    g_cmap = nullptr;
    g_cmap_bytes = 0;
  }
}

namespace {

struct CohortMapped {
  void* p = nullptr;
  bool own = false;
  ~CohortMapped() {
    if (own) {
      cudaFreeHost(p);
    } else if (p) {
      std::lock_guard<std::mutex> lk(g_cmap_mu);
      g_cmap_busy = false;
    }
  }
  Status take(size_t bytes) {
    {
      std::lock_guard<std::mutex> lk(g_cmap_mu);
      if (!g_cmap_busy) {
        if (g_cmap_bytes < bytes) {
          // with headroom (pinning host memory costs milliseconds to a second): a small
          // first call does not force a larger one to pin again
          const size_t want = std::max<size_t>(bytes, (size_t)64 << 20);
          if (g_cmap) cudaFreeHost(g_cmap);
          g_cmap = nullptr;
          g_cmap_bytes = 0;
          SG_CUDA(cudaHostAlloc(&g_cmap, want, cudaHostAllocMapped));
          g_cmap_bytes = want;
        }
        g_cmap_busy = true;
        p = g_cmap;
        return Status();
      }
    }
    own = true;
    SG_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocMapped));
    return Status();
  }
};

// The streamed build of every cohort's GRM (MIXED fits): the .bed streams in by marker
// chunks on a copy stream; as each chunk lands, one launch counts every cohort's alleles
// and missing calls of its markers (into host-mapped memory), the host applies each
// cohort's marker QC (fit_null.rs:209-222) to them and writes where each passing marker
// goes (the next row of that cohort), and one launch gathers the chunk's rows into every
// cohort's handle — all under the PCIe-bound transfer.  Rows are then every QC-passing
// marker in .bed order; grm_stream_rows_finish draws the variance-ratio candidates among
// them and keeps them in place with zero metadata, so the tensor-core products are
// bit-identical to those of a handle holding only the GRM markers (the sequential path).
Status stream_cohorts(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot, int dev,
                      double min_maf, double max_missing, uint64_t seed, DevBuf& d_bed,
                      std::vector<CohortJob>& jobs) {
  const int64_t bpm = (n_fam + 3) / 4;
  const int k = (int)jobs.size();
  PhaseTimer tm;
  std::vector<int32_t> all;
  std::vector<int64_t> offs((size_t)k), ns((size_t)k);
  for (int c = 0; c < k; ++c) {
    std::vector<int32_t> sv;
    bool identity = true;
    SG_TRY(check_subset(jobs[(size_t)c].sidx, jobs[(size_t)c].n, n_fam, sv, identity));
    offs[(size_t)c] = (int64_t)all.size();
    ns[(size_t)c] = jobs[(size_t)c].n;
    all.insert(all.end(), sv.begin(), sv.end());
    all.resize((size_t)round_up((int64_t)all.size(), 16), 0);
  }
  CohortMapped mp;
  const size_t cnt_bytes = (size_t)k * m_tot * 2 * sizeof(long long);
  SG_TRY(mp.take(cnt_bytes + (size_t)m_tot * k * sizeof(int32_t)));
  long long* cnt_h = static_cast<long long*>(mp.p);
  int32_t* map_h = reinterpret_cast<int32_t*>(static_cast<char*>(mp.p) + cnt_bytes);
  void* mp_dev = nullptr;
  SG_CUDA(cudaHostGetDevicePointer(&mp_dev, mp.p, 0));
  long long* cnt_d = static_cast<long long*>(mp_dev);
  const int32_t* map_d = reinterpret_cast<const int32_t*>(static_cast<char*>(mp_dev) + cnt_bytes);
  std::vector<std::vector<int64_t>> pass((size_t)k);
  cudaStream_t cp = nullptr, kst = nullptr;
  std::vector<cudaEvent_t> ev;
  cudaEvent_t counted = nullptr;
  DevBuf d_sidx, d_offs, d_ns;
  auto body = [&]() -> Status {
    SG_CUDA(cudaStreamCreateWithFlags(&cp, cudaStreamNonBlocking));
    SG_CUDA(cudaStreamCreateWithFlags(&kst, cudaStreamNonBlocking));
    SG_CUDA(cudaEventCreateWithFlags(&counted, cudaEventDisableTiming));
    SG_TRY(d_sidx.reserve(all.size() * 4));
    SG_TRY(d_offs.reserve((size_t)k * 8));
    SG_TRY(d_ns.reserve((size_t)k * 8));
    // the sample lists ahead of the .bed on the copy engine
    SG_CUDA(cudaMemcpyAsync(d_sidx.ptr, all.data(), all.size() * 4, cudaMemcpyHostToDevice, kst));
    SG_CUDA(cudaMemcpyAsync(d_offs.ptr, offs.data(), (size_t)k * 8, cudaMemcpyHostToDevice, kst));
    SG_CUDA(cudaMemcpyAsync(d_ns.ptr, ns.data(), (size_t)k * 8, cudaMemcpyHostToDevice, kst));
    SG_CUDA(cudaStreamSynchronize(kst));
    constexpr int kChunks = 32;
    const int64_t per = std::max<int64_t>(1, ceil_div(m_tot, (int64_t)kChunks));
    uint8_t* dst = d_bed.as<uint8_t>();
    std::vector<std::pair<int64_t, int64_t>> spans;
    for (int64_t j0 = 0; j0 < m_tot; j0 += per) {
      const int64_t j1 = std::min(m_tot, j0 + per);
      const size_t lo = j0 == 0 ? 0 : (size_t)(3 + j0 * bpm);
      const size_t hi = j1 == m_tot ? bed_len : (size_t)(3 + j1 * bpm);
      SG_CUDA(cudaMemcpyAsync(dst + lo, bed + lo, hi - lo, cudaMemcpyHostToDevice, cp));
      cudaEvent_t e = nullptr;
      SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ev.push_back(e);
      SG_CUDA(cudaEventRecord(e, cp));
      spans.emplace_back(j0, j1);
    }
    // the handles (room for every marker) while the first chunks land
    {
      std::vector<std::thread> th;
      for (int c = 0; c < k; ++c)
        th.emplace_back([&, c]() {
          cudaSetDevice(dev);
          CohortJob& j = jobs[(size_t)c];
          j.rc = grm_shell_create_cap(dev, j.n, m_tot, &j.h).code;
          if (j.rc != SAIGE_OK) j.err = saige_last_error();
          j.af.resize((size_t)m_tot);
          j.mac.resize((size_t)m_tot);
          j.nv.resize((size_t)m_tot);
          pass[(size_t)c].reserve((size_t)m_tot);
        });
      for (auto& t : th) t.join();
    }
    for (int c = 0; c < k; ++c)
      if (jobs[(size_t)c].rc != SAIGE_OK)
        return fail(jobs[(size_t)c].rc, "cohort %d: %s", c, jobs[(size_t)c].err.c_str());
    tm.mark(" handles");
    std::vector<std::pair<int, int64_t>> degenerate;
    for (size_t i = 0; i < spans.size(); ++i) {
      const int64_t j0 = spans[i].first, j1 = spans[i].second;
      SG_CUDA(cudaStreamWaitEvent(kst, ev[i], 0));
      SG_CUDA(launch_bed_count_cohorts(dst, bpm, j0, j1 - j0, d_sidx.as<int32_t>(),
                                       d_offs.as<int64_t>(), d_ns.as<int64_t>(), k, m_tot, cnt_d,
                                       kst));
      SG_CUDA(cudaEventRecord(counted, kst));
      SG_CUDA(cudaEventSynchronize(counted));
      degenerate.clear();
      for (int c = 0; c < k; ++c) {
        CohortJob& jb = jobs[(size_t)c];
        stats_from_counts(cnt_h + 2 * ((size_t)c * m_tot + j0), j1 - j0, jb.n, jb.af.data() + j0,
                          jb.mac.data() + j0, jb.nv.data() + j0);
        std::vector<int64_t>& ps = pass[(size_t)c];
        for (int64_t j = j0; j < j1; ++j) {
          int32_t r = -1;
          if (marker_qc_pass(jb.af[(size_t)j], jb.nv[(size_t)j], jb.n, min_maf, max_missing)) {
            r = (int32_t)ps.size();
            ps.push_back(j);
            const double pj = jb.af[(size_t)j];
            if (!(sqrt(2.0 * pj * (1.0 - pj)) > 1e-10)) degenerate.emplace_back(c, (int64_t)r);
          }
          map_h[(size_t)j * k + c] = r;
        }
      }
      for (int c0 = 0; c0 < k; c0 += kCohortsPerLaunch) {
        CohortSet set{};
        set.n = std::min(kCohortsPerLaunch, k - c0);
        for (int q = 0; q < set.n; ++q) {
          const saige_grm* h = jobs[(size_t)(c0 + q)].h;
          set.c[q] = CohortRows{h->geno, map_d + (c0 + q), (int64_t)k, h->wpr, h->n,
                                offs[(size_t)(c0 + q)]};
        }
        SG_CUDA(launch_bed_gather_cohorts(dst, bpm, j0, j1 - j0, d_sidx.as<int32_t>(), set, kst));
      }
      // a zero standardised column: codes 11, as grm_blank_degenerate_rows does
      for (const auto& dg : degenerate) {
        const saige_grm* h = jobs[(size_t)dg.first].h;
        SG_CUDA(cudaMemsetAsync(h->geno + (size_t)dg.second * h->wpr, 0xFF, (size_t)h->wpr * 4, kst));
      }
    }
    SG_CUDA(cudaStreamSynchronize(kst));
    SG_CUDA(cudaStreamSynchronize(cp));
    tm.mark(" upload+counts+gather");
    return Status();
  };
  Status s = body();
  if (cp) cudaStreamSynchronize(cp);
  if (kst) cudaStreamSynchronize(kst);
  {
    ReleaseScope idle(ReleaseMode::kIdle, nullptr);  // both streams have drained
    d_sidx.release();
    d_offs.release();
    d_ns.release();
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  if (counted) cudaEventDestroy(counted);
  if (cp) cudaStreamDestroy(cp);
  if (kst) cudaStreamDestroy(kst);
  SG_TRY(s);
  // variance-ratio candidates, padding rows and metadata of each cohort (in parallel)
  {
    std::vector<std::thread> th;
    for (int c = 0; c < k; ++c)
      th.emplace_back([&, c]() {
        cudaSetDevice(dev);
        CohortJob& j = jobs[(size_t)c];
        std::vector<int64_t> vidx;
        j.rc = grm_stream_rows_finish(j.h, pass[(size_t)c], j.af.data(), j.mac.data(), seed, vidx)
                   .code;
        if (j.rc != SAIGE_OK) j.err = saige_last_error();
        j.m_grm = j.h->m_eff;
        j.have_stats = true;
      });
    for (auto& t : th) t.join();
  }
  for (int c = 0; c < k; ++c)
    if (jobs[(size_t)c].rc != SAIGE_OK)
      return fail(jobs[(size_t)c].rc, "cohort %d: %s", c, jobs[(size_t)c].err.c_str());
  tm.mark(" finish");
  return Status();
}

// Every cohort's marker selection and GRM handle, with the packed rows of all of them
// from one pass over the device .bed (each raw row staged once for all cohorts).
Status build_handles(const uint8_t* d_bed, int64_t n_fam, int64_t m_tot, int dev, double min_maf,
                     double max_missing, uint64_t seed, const SampleLists& lists,
                     std::vector<CohortJob>& jobs) {
  const int k = (int)jobs.size();
  const int64_t bpm = (n_fam + 3) / 4;
  PhaseTimer tm;
  std::vector<int32_t> row_of((size_t)k * m_tot, -1);
  // selection, handle and metadata of each cohort on its own host thread (a few ms of
  // host work and uploads each)
  auto prepare = [&](int c) {
    CohortJob& j = jobs[(size_t)c];
    cudaSetDevice(dev);
    j.gidx.assign((size_t)m_tot, 0);
    std::vector<int64_t> vidx((size_t)m_tot);
    int64_t m_grm = 0, m_vr = 0;
    j.rc = saige_select_grm_markers(j.af.data(), j.mac.data(), j.nv.data(), m_tot, j.n, min_maf,
                                    max_missing, seed, j.gidx.data(), &m_grm, vidx.data(), &m_vr);
    if (j.rc == SAIGE_OK) {
      j.gidx.resize((size_t)m_grm);
      j.m_grm = m_grm;
      j.gaf.resize((size_t)m_grm);
      for (int64_t r = 0; r < m_grm; ++r) {
        j.gaf[(size_t)r] = j.af[(size_t)j.gidx[(size_t)r]];
        row_of[(size_t)c * m_tot + (size_t)j.gidx[(size_t)r]] = (int32_t)r;
      }
      j.rc = grm_shell_create(dev, j.n, m_grm, j.gaf.data(), &j.h).code;
    }
    if (j.rc != SAIGE_OK) j.err = saige_last_error();
  };
  {
    std::vector<std::thread> th;
    for (int c = 0; c < k; ++c) th.emplace_back(prepare, c);
    for (auto& t : th) t.join();
  }
  for (int c = 0; c < k; ++c)
    if (jobs[(size_t)c].rc != SAIGE_OK)
      return fail(jobs[(size_t)c].rc, "cohort %d: %s", c, jobs[(size_t)c].err.c_str());
  tm.mark(" select+alloc");
  cudaStream_t st = nullptr;
  DevBuf d_rows;
  auto body = [&]() -> Status {
    SG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    SG_TRY(d_rows.reserve(row_of.size() * 4));
    SG_CUDA(cudaMemcpyAsync(d_rows.ptr, row_of.data(), row_of.size() * 4, cudaMemcpyHostToDevice,
                            st));
    for (int c0 = 0; c0 < k; c0 += kCohortsPerLaunch) {
      CohortSet set{};
      set.n = std::min(kCohortsPerLaunch, k - c0);
      for (int i = 0; i < set.n; ++i) {
        const saige_grm* h = jobs[(size_t)(c0 + i)].h;
        set.c[i] = CohortRows{h->geno, d_rows.as<int32_t>() + (size_t)(c0 + i) * m_tot, 1,
                              h->wpr, h->n, lists.offs[(size_t)(c0 + i)]};
      }
      SG_CUDA(launch_bed_gather_cohorts(d_bed, bpm, 0, m_tot, lists.d_sidx.as<int32_t>(), set, st));
    }
    SG_CUDA(cudaStreamSynchronize(st));
    return Status();
  };
  Status s = body();
  if (st) cudaStreamSynchronize(st);
  {
    ReleaseScope idle(ReleaseMode::kIdle, nullptr);  // the stream has drained
    d_rows.release();
  }
  if (st) cudaStreamDestroy(st);
  SG_TRY(s);
  tm.mark(" gather");
  for (int c = 0; c < k; ++c) SG_TRY(grm_shell_finish(jobs[(size_t)c].h, jobs[(size_t)c].gaf.data()));
  tm.mark(" finish");
  return Status();
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
    Status hs = check_bed_header(bed, bed_len, n_fam, m_tot);
    if (!hs.ok()) return hs.code;
    saige_ai_reml_config cf;
    if (cfg) cf = *cfg;
    else saige_ai_reml_config_default(&cf);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(SAIGE_ECUDA, "no CUDA device").code;
    const auto t0 = std::chrono::steady_clock::now();
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
    DevBuf d_bed;
    Status s = d_bed.reserve(bed_len);
    if (!s.ok()) return s.code;
    const int64_t bpm = (n_fam + 3) / 4;
    SampleLists lists;
    auto drop_handles = [&]() {
      for (CohortJob& j : jobs)
        if (j.h) {
          grm_shell_destroy(j.h);
          j.h = nullptr;
        }
    };
    PhaseTimer tm;
    if (concurrent && bpm <= 200 * 1024 && cf.precision == SAIGE_PREC_MIXED) {
      s = stream_cohorts(bed, bed_len, n_fam, m_tot, dev, min_maf, max_missing, cf.seed, d_bed,
                         jobs);
      if (!s.ok()) {
        drop_handles();
        return s.code;
      }
    } else if (concurrent && bpm <= 200 * 1024) {
      // FP32 fits: the rows must be the GRM markers only (an FP32 product's grouping of
      // its sums follows the row count), so the selection waits for all the counts
      s = upload_and_count(bed, bed_len, n_fam, m_tot, d_bed, jobs, lists);
      tm.mark("upload+counts");
      if (s.ok())
        s = build_handles(d_bed.as<uint8_t>(), n_fam, m_tot, dev, min_maf, max_missing, cf.seed,
                          lists, jobs);
      lists.d_sidx.release();
      if (!s.ok()) {
        drop_handles();
        return s.code;
      }
    } else if (cudaMemcpy(d_bed.ptr, bed, bed_len, cudaMemcpyHostToDevice) != cudaSuccess) {
      return fail(SAIGE_ECUDA, "bed upload failed: %s", cudaGetErrorString(cudaGetLastError())).code;
    }
    const uint8_t* db = d_bed.as<uint8_t>();
    if (concurrent) {
      // a pool of host threads, each with its cohorts' streams: half the hardware threads
      // (at least two; a fit's host thread spins on its stream's syncs, so one per
      // cohort oversubscribed the cores and stalled whole runs), largest cohorts first
      std::vector<int32_t> order((size_t)n_cohorts);
      for (int32_t c = 0; c < n_cohorts; ++c) order[(size_t)c] = c;
      std::stable_sort(order.begin(), order.end(),
                       [&](int32_t a, int32_t b) { return jobs[(size_t)a].n > jobs[(size_t)b].n; });
      const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
      const int32_t workers = std::min<int32_t>(n_cohorts, (int32_t)std::max(2u, hw / 2));
      std::atomic<int32_t> next{0};
      auto worker = [&]() {
        for (int32_t i = next++; i < n_cohorts; i = next++)
          run_cohort(dev, db, bed_len, n_fam, m_tot, p, trait, min_maf, max_missing, &cf,
                     jobs[(size_t)order[(size_t)i]]);
      };
      std::vector<std::thread> th;
      th.reserve((size_t)workers);
      for (int32_t w = 0; w < workers; ++w) th.emplace_back(worker);
      for (auto& t : th) t.join();
      tm.mark("fits");
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
