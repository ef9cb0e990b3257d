// Internal engine of the fit-null library: the GRM handle, the GRM product
// dispatch and the PCG driver shared by the C ABI and the AI-REML loop.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "kernels_vec.cuh"

namespace saige {

// Growable device buffer.  Blocks of at least kCacheMinBytes go through a per-device
// cache: release() keeps them (after synchronising their device, as cudaFree would)
// and reserve() reuses a cached block of the same device of 1 to 1.25 times the size,
// so that repeated fits of one cohort shape do not map and unmap tens of GB each
// time.  release_cached_blocks() hands the cache back to the driver.
//
// Inside a ReleaseScope on the calling thread, release() knows more about the work
// that may still use a block: kStream — all of it is ordered on one stream, which is
// synchronised instead of the whole device; kIdle — none is in flight.  Such blocks
// are cached whatever their size (cudaFree would synchronise the device), so that
// fits running side by side on their own streams do not wait for one another.
constexpr size_t kCacheMinBytes = (size_t)1 << 20;

enum class ReleaseMode { kDevice, kStream, kIdle };

struct ReleaseScope {
  ReleaseMode prev_mode;
  cudaStream_t prev_stream;
  ReleaseScope(ReleaseMode mode, cudaStream_t stream);
  ~ReleaseScope();
  ReleaseScope(const ReleaseScope&) = delete;
  ReleaseScope& operator=(const ReleaseScope&) = delete;
};

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  int dev = -1;
  Status reserve(size_t want);
  void release();
  template <class T> T* as() const { return static_cast<T*>(ptr); }
  ~DevBuf() { release(); }
};

void release_cached_blocks();
// Frees the sub-cohort build's host-mapped block unless a call is using it (cohorts.cu).
void release_cohort_mapped();

// Makes device d current for the scope and gives the caller's device back at the
// end, on every return path.  ok is false when d could not be made current.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      (void)cudaGetLastError();
    }
    if (prev != d && cudaSetDevice(d) != cudaSuccess) {
      ok = false;
      (void)cudaGetLastError();
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

struct TcPlan;  // tensor-core path state (kernels_tc.cu)

// Selects (want >= 0) or checks (want < 0: the current) device; fails unless it is sm_100.
Status pick_device(int32_t want, int* dev);
// PLINK .bed magic, SNP-major mode and size (plink.rs:80-98).
Status check_bed_header(const uint8_t* hdr, size_t bed_len, int64_t n_fam, int64_t m_tot);
// MarkerData::compute_af (saige-geno/src/traits.rs:42-54) from exact counts of n
// samples: cnt[2j] alt-allele count, cnt[2j + 1] missing calls of marker j; the same
// f64 operations on the same integers as the reference's dosage sums.
void stats_from_counts(const long long* cnt, int64_t m, int64_t n, double* af, double* mac,
                       int64_t* n_valid);
// Validates a sample subset (NULL = all n_fam samples in order).
Status check_subset(const int64_t* sidx, int64_t n, int64_t n_fam, std::vector<int32_t>& out,
                    bool& identity);
// Gathers .bed rows (device-resident .bed) into packed rows of wpr words and/or
// per-row {alt count, missing count}; synchronises the stream.
Status bed_gather_dev(const uint8_t* bed_dev, int64_t n_fam, const std::vector<int64_t>& rows,
                      const std::vector<int32_t>& sidx, bool identity, int64_t n,
                      uint32_t* geno_out, int64_t wpr, int64_t* counts_dev, cudaStream_t st);

// The fit-null GRM handle built while the .bed (pinned host memory, bed_len bytes)
// streams into d_bed: marker counts into af/mac/nv (length m_tot), the QC of
// fit_null.rs:209-222, the variance-ratio candidates into vidx, m_grm = the GRM's M.
// The handle's rows are all QC-passing markers; the candidates' rows carry
// 2p = 1/s = 0 and m_eff = m_grm.  For MIXED products only.
Status stream_fit_null_grm(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                           const int64_t* sample_idx, int64_t n, double min_maf,
                           double max_missing, uint64_t seed, DevBuf& d_bed,
                           std::vector<double>& af, std::vector<double>& mac,
                           std::vector<int64_t>& nv, std::vector<int64_t>& vidx, int64_t& m_grm,
                           saige_grm** out);

}  // namespace saige

struct saige_grm {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::recursive_mutex mu;
  int64_t n = 0, n_pad = 0, wpr = 0;  // samples, padded samples, 32-bit words per row
  int64_t m = 0, m_pad = 0;           // marker rows, padded marker rows
  // markers that enter K (the 1/M of every product): m, less the rows a streamed
  // build kept in place with 2p = 1/s = 0 (variance-ratio candidates)
  int64_t m_eff = 0;
  uint32_t* geno = nullptr;           // m_pad x wpr packed 2-bit codes (in geno_buf)
  saige::DevBuf geno_buf;
  saige::DevBuf meta_buf;             // holds zlut, two_p and inv_s
  float4* zlut = nullptr;             // per marker: f32 z for codes 00,01,10,11
  double* two_p = nullptr;            // per marker 2p (0 for padding)
  double* inv_s = nullptr;            // per marker 1/sqrt(2p(1-p)) (0 when degenerate / padding)
  // FP32 product workspace
  saige::DevBuf v32, u32, ypart;
  int n_splits = 1;
  // tensor-core product state
  saige::TcPlan* tc = nullptr;
  // generic workspaces
  saige::DevBuf ws_vec, ws_red, ws_cols, ws_io;
  // Leave-one-chromosome-out: while `masked`, products skip the markers flagged in
  // excl (m_pad bytes, 1 = left out) and scale by 1/m_active.  Set and cleared only
  // inside saige_fit_loco, under mu.
  bool masked = false;
  int64_t m_active = 0;
  saige::DevBuf excl;
  // statistics
  int64_t n_kv = 0, n_kv_launches = 0;
  int64_t n_fits = 0;  // AI-REML fits started on the handle (the missing-call lists' trigger)
  bool profiling = false;
  saige_grm_stats stats{};
};

namespace saige {

// A handle for n samples and m marker rows (allele frequencies af) whose packed rows
// the caller writes — rows [m, m_pad) are already coded 11 — then grm_shell_finish
// recodes the zero-variance rows and drains the handle's stream.  For builds that fill
// several handles from one pass over the .bed (the sub-cohorts).
Status grm_shell_create(int dev, int64_t n, int64_t m, const double* af, saige_grm** out);
Status grm_shell_finish(saige_grm* h, const double* af);
void grm_shell_destroy(saige_grm* h);
// A handle with room for rows_cap marker rows and no metadata yet, for a streamed
// build: the caller gathers the QC-passing markers into rows 0, 1, ... as the .bed
// lands, then grm_stream_rows_finish(pass = their .bed indices, af and mac over all
// markers) draws the variance-ratio candidates among them (kept in place with 2p = 1/s
// = 0, so that integer products are those of a handle holding only the GRM markers),
// codes the padding rows 11, uploads the metadata and sets m, m_pad, m_eff (the GRM's
// M).  vidx receives the candidates' .bed indices.
Status grm_shell_create_cap(int dev, int64_t n, int64_t rows_cap, saige_grm** out);
Status grm_stream_rows_finish(saige_grm* h, const std::vector<int64_t>& pass, const double* af,
                              const double* mac, uint64_t seed, std::vector<int64_t>& vidx);
// fit_null.rs:209-222's marker QC over n samples (MAF and call rate).
bool marker_qc_pass(double af, int64_t n_valid, int64_t n, double min_maf, double max_missing);

// Kv for q columns of v (ld = h->n_pad, padding rows zero) into kp.
// active (host, length q, may be NULL) selects columns; others are skipped.
Status grm_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                   int precision, cudaStream_t st);

struct PcgRun {
  // inputs (device, ld = n_pad)
  const double* b = nullptr;
  const double* x0 = nullptr;
  const double* ax0 = nullptr; // Sigma x0 when the caller knows it (no product for r0)
  const double* wv = nullptr;  // wmax (fit-null form) or w (score-test form)
  const double* d = nullptr;   // Jacobi diagonal
  double tau0 = 1.0, tau1 = 0.0;
  bool w_inverse = true;       // fit-null operator tau0 v/w + tau1 K v
  int q = 1;
  double tol = 1e-5;
  int max_iter = 500;
  int precision = SAIGE_PREC_FP32;
  bool force_step = false;     // warm starts: at least one CG step per column
  // outputs
  double* x = nullptr;         // device n_pad x q
  double* r_out = nullptr;     // optional: the final residual b - Sigma x (device n_pad x q)
  // optional: K x kept beside x from the products K p (device n_pad x q); kx0 = K x0
  // when x0 and ax0 are given.  kx_valid is false when no product was formed (tau1 = 0).
  double* kx = nullptr;
  const double* kx0 = nullptr;
  bool kx_valid = false;
  // optional: n_extra more columns (device, ld apart) multiplied by K in the solve's
  // first product launch, the product into extra_out; a separate launch when none runs
  const double* extra_in = nullptr;
  double* extra_out = nullptr;
  int n_extra = 0;
  // optional: the search directions p of the first keep_cols columns, with their
  // K-images, copied after each product into keep_p / keep_kp (ld apart) while the
  // column is active, up to keep_cap vectors; kept = how many on return
  double* keep_p = nullptr;
  double* keep_kp = nullptr;
  int keep_cols = 0, keep_cap = 0, kept = 0;
  std::vector<int32_t> iters, state;
  std::vector<double> resid;
  int64_t total_iters = 0;
};

// Block PCG with per-column masks (decomposition.rs:212-298 per column).
Status pcg_run(saige_grm* h, PcgRun& run, cudaStream_t st);

// Device scratch carved from the handle's workspaces.
struct PcgScratch {
  double *r, *z, *p, *ap, *kp;
  double* partial;
  double* small;  // >= 4*q
  PcgCols cols;
};
Status pcg_scratch(saige_grm* h, int q, PcgScratch& s);

}  // namespace saige
