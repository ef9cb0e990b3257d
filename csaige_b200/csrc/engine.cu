// GRM handle lifecycle, GRM product dispatch, PCG driver and the C ABI.
#include <math.h>
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <vector>

#include "engine.cuh"
#include "kernels.cuh"
#include "kernels_tc.cuh"
#include "warm.cuh"
#include "rng.hpp"

namespace saige {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static std::atomic<int64_t> g_launches{0};

void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }
void count_launches(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
int64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }

Status fail(int32_t code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return Status(code);
}

namespace {
struct CachedBlock {
  int dev;
  size_t bytes;
  void* ptr;
};
std::mutex g_cache_mu;
std::vector<CachedBlock> g_cache;

// the streamed fit-null build's host-mapped block (see stream_fit_null_grm)
std::mutex g_mapped_mu;
void* g_mapped = nullptr;
size_t g_mapped_bytes = 0;
bool g_mapped_busy = false;

// Takes the smallest cached block of `dev` with want <= bytes <= 1.25 want.
bool cache_take(int dev, size_t want, void** ptr, size_t* bytes) {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  size_t best = g_cache.size();
  for (size_t i = 0; i < g_cache.size(); ++i) {
    const CachedBlock& b = g_cache[i];
    if (b.dev == dev && b.bytes >= want && b.bytes <= want + want / 4 &&
        (best == g_cache.size() || b.bytes < g_cache[best].bytes))
      best = i;
  }
  if (best == g_cache.size()) return false;
  *ptr = g_cache[best].ptr;
  *bytes = g_cache[best].bytes;
  g_cache.erase(g_cache.begin() + (std::ptrdiff_t)best);
  return true;
}

// Frees every cached block of `dev` (all devices when dev < 0); returns how many.
size_t cache_flush(int dev) {
  std::vector<CachedBlock> out;
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (size_t i = 0; i < g_cache.size();) {
      if (dev < 0 || g_cache[i].dev == dev) {
        out.push_back(g_cache[i]);
        g_cache.erase(g_cache.begin() + (std::ptrdiff_t)i);
      } else {
        ++i;
      }
    }
  }
  int cur = -1;
  cudaGetDevice(&cur);
  for (const CachedBlock& b : out) {
    cudaSetDevice(b.dev);
    cudaFree(b.ptr);
  }
  if (cur >= 0) cudaSetDevice(cur);
  return out.size();
}
}  // namespace

void release_cached_blocks() {
  cache_flush(-1);
  // the sub-cohort build's host-mapped block, unless a build is using it
  release_cohort_mapped();
  // the streamed build's host-mapped block, unless a build is using it
  std::lock_guard<std::mutex> lk(g_mapped_mu);
  if (g_mapped && !g_mapped_busy) {
    cudaFreeHost(g_mapped);
    g_mapped = nullptr;
    g_mapped_bytes = 0;
  }
}

Status DevBuf::reserve(size_t want) {
  if (want <= bytes) return Status();
  release();
  if (want == 0) return Status();
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) d = 0;
  if (cache_take(d, want, &ptr, &bytes)) {
    dev = d;
    return Status();
  }
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e == cudaErrorMemoryAllocation && cache_flush(d) > 0) {
    (void)cudaGetLastError();
    e = cudaMalloc(&ptr, want);
  }
  if (e != cudaSuccess) {
    ptr = nullptr;
    bytes = 0;
    (void)cudaGetLastError();
    return fail(SAIGE_ENOMEM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
  }
  bytes = want;
  dev = d;
  return Status();
}

namespace {
thread_local ReleaseMode tl_release_mode = ReleaseMode::kDevice;
thread_local cudaStream_t tl_release_stream = nullptr;
}  // namespace

ReleaseScope::ReleaseScope(ReleaseMode mode, cudaStream_t stream)
    : prev_mode(tl_release_mode), prev_stream(tl_release_stream) {
  tl_release_mode = mode;
  tl_release_stream = stream;
}

ReleaseScope::~ReleaseScope() {
  tl_release_mode = prev_mode;
  tl_release_stream = prev_stream;
}

void DevBuf::release() {
  if (ptr) {
    const ReleaseMode mode = tl_release_mode;
    if (dev >= 0 && (bytes >= kCacheMinBytes || mode != ReleaseMode::kDevice)) {
      // as cudaFree would, wait for the work that may still use the block before it
      // can be reused: the device's, the scope's stream, or none when it is idle
      if (mode == ReleaseMode::kStream) {
        cudaStreamSynchronize(tl_release_stream);
      } else if (mode == ReleaseMode::kDevice) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (cur != dev) cudaSetDevice(dev);
        cudaDeviceSynchronize();
        if (cur >= 0 && cur != dev) cudaSetDevice(cur);
      }
      std::lock_guard<std::mutex> lk(g_cache_mu);
      g_cache.push_back(CachedBlock{dev, bytes, ptr});
    } else {
      cudaFree(ptr);
    }
  }
  ptr = nullptr;
  bytes = 0;
  dev = -1;
}

// ---------------------------------------------------------------------------
// device selection
// ---------------------------------------------------------------------------
Status pick_device(int32_t want, int* dev) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    (void)cudaGetLastError();
    return fail(SAIGE_ECUDA, "no CUDA device available (%s)",
                e == cudaSuccess ? "count = 0" : cudaGetErrorString(e));
  }
  int d = want;
  if (d < 0) SG_CUDA(cudaGetDevice(&d));
  if (d >= count) return fail(SAIGE_EINVAL, "device %d out of range (%d devices)", d, count);
  // two attribute queries (a full cudaGetDeviceProperties costs milliseconds per call)
  int major = 0, minor = 0;
  SG_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d));
  SG_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, d));
  if (major != 10 || minor != 0)
    return fail(SAIGE_ECUDA, "device %d is sm_%d%d; this library is built for sm_100a only", d,
                major, minor);
  SG_CUDA(cudaSetDevice(d));
  if (dev) *dev = d;
  return Status();
}


// ---------------------------------------------------------------------------
// per-marker metadata (pcg.rs:101-122 arithmetic, done on the host in f64)
// ---------------------------------------------------------------------------
static void marker_meta(const double* af, int64_t m, int64_t m_pad, std::vector<float4>& zl,
                        std::vector<double>& tp, std::vector<double>& is) {
  zl.assign((size_t)m_pad, make_float4(0.f, 0.f, 0.f, 0.f));
  tp.assign((size_t)m_pad, 0.0);
  is.assign((size_t)m_pad, 0.0);
  for (int64_t j = 0; j < m; ++j) {
    const double p = af[j];
    const double denom = sqrt(2.0 * p * (1.0 - p));
    if (!(denom > 1e-10)) continue;  // OnTheFlyGrm leaves the column at 0
    const double mean = 2.0 * p;
    // codes 00 -> 2, 01 -> missing (mean, so exactly 0), 10 -> 1, 11 -> 0
    zl[j] = make_float4((float)((2.0 - mean) / denom), 0.0f, (float)((1.0 - mean) / denom),
                        (float)((0.0 - mean) / denom));
    tp[j] = mean;
    is[j] = 1.0 / denom;
  }
}

// zlut, two_p and inv_s for `rows` marker rows in one block (from the buffer cache)
static Status grm_alloc_meta(saige_grm* h, int64_t rows) {
  SG_TRY(h->meta_buf.reserve((size_t)rows * (sizeof(float4) + 2 * sizeof(double))));
  h->zlut = h->meta_buf.as<float4>();
  h->two_p = reinterpret_cast<double*>(h->zlut + rows);
  h->inv_s = h->two_p + rows;
  return Status();
}

static Status grm_alloc(saige_grm* h, int64_t n, int64_t m) {
  h->n = n;
  h->n_pad = round_up(std::max<int64_t>(n, 1), kSamplePad);
  h->wpr = h->n_pad / 16;
  h->m = m;
  h->m_eff = m;
  h->m_pad = round_up(std::max<int64_t>(m, 1), kMarkerPad);
  SG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  SG_TRY(h->geno_buf.reserve((size_t)h->m_pad * h->wpr * 4));
  h->geno = h->geno_buf.as<uint32_t>();
  SG_TRY(grm_alloc_meta(h, h->m_pad));
  // padding rows: all codes 11 (genotype 0, not missing); their 1/s and 2p are 0
  SG_CUDA(cudaMemsetAsync(h->geno + (size_t)m * h->wpr, 0xFF,
                          (size_t)(h->m_pad - m) * h->wpr * 4, h->stream));
  h->n_splits = fp32_z_splits(h->n_pad, h->m_pad);
  return Status();
}

static Status grm_upload_meta(saige_grm* h, const double* af) {
  std::vector<float4> zl;
  std::vector<double> tp, is;
  marker_meta(af, h->m, h->m_pad, zl, tp, is);
  // on the handle's stream: a legacy-stream copy from pageable memory may still be in
  // flight when it returns, and the handle's (non-blocking) stream would not wait for it
  SG_CUDA(cudaMemcpyAsync(h->zlut, zl.data(), zl.size() * sizeof(float4), cudaMemcpyHostToDevice,
                          h->stream));
  SG_CUDA(cudaMemcpyAsync(h->two_p, tp.data(), tp.size() * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
  SG_CUDA(cudaMemcpyAsync(h->inv_s, is.data(), is.size() * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
  SG_CUDA(cudaStreamSynchronize(h->stream));  // the host vectors go out of scope
  return Status();
}

// A marker whose standardised column is zero (denominator <= 1e-10, pcg.rs:108)
// contributes nothing; its row is re-coded 11 so no kernel does work for its
// missing calls.
static Status grm_blank_degenerate_rows(saige_grm* h, const double* af) {
  for (int64_t j = 0; j < h->m; ++j) {
    const double denom = sqrt(2.0 * af[j] * (1.0 - af[j]));
    if (!(denom > 1e-10))
      SG_CUDA(cudaMemsetAsync(h->geno + (size_t)j * h->wpr, 0xFF, (size_t)h->wpr * 4, h->stream));
  }
  return Status();
}

static void grm_free(saige_grm* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  // every buffer of the handle is used on its stream only, now idle
  ReleaseScope idle(ReleaseMode::kIdle, nullptr);
  tc_destroy(h);
  h->v32.release();
  h->u32.release();
  h->ypart.release();
  h->ws_vec.release();
  h->ws_red.release();
  h->ws_cols.release();
  h->ws_io.release();
  h->geno_buf.release();
  h->geno = nullptr;
  h->meta_buf.release();
  h->zlut = nullptr;
  h->two_p = h->inv_s = nullptr;
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

Status check_bed_header(const uint8_t* hdr, size_t bed_len, int64_t n_fam, int64_t m_tot) {
  if (bed_len < 3) return fail(SAIGE_EBED, "Bed file too small");
  if (hdr[0] != 0x6C || hdr[1] != 0x1B) return fail(SAIGE_EBED, "Invalid PLINK bed file magic number");
  if (hdr[2] != 0x01)
    return fail(SAIGE_EBED, "Only SNP-major bed files are supported (mode byte = 0x01)");
  const int64_t bpm = (n_fam + 3) / 4;
  if ((int64_t)bed_len < 3 + bpm * m_tot)
    return fail(SAIGE_EBED, "Bed file too small: expected at least %lld bytes, got %zu",
                (long long)(3 + bpm * m_tot), bed_len);
  return Status();
}

Status check_subset(const int64_t* sidx, int64_t n, int64_t n_fam,
                           std::vector<int32_t>& out, bool& identity) {
  identity = true;
  if (n <= 0) return fail(SAIGE_EINVAL, "n must be positive");
  if (n_fam > INT32_MAX) return fail(SAIGE_EINVAL, "n_fam exceeds 2^31-1");
  if (!sidx) {
    if (n != n_fam) return fail(SAIGE_EINVAL, "n (%lld) != n_fam (%lld) without sample_idx",
                                (long long)n, (long long)n_fam);
    return Status();
  }
  out.resize((size_t)n);
  for (int64_t k = 0; k < n; ++k) {
    if (sidx[k] < 0 || sidx[k] >= n_fam)
      return fail(SAIGE_EINVAL, "sample_idx[%lld] = %lld out of range", (long long)k,
                  (long long)sidx[k]);
    out[(size_t)k] = (int32_t)sidx[k];
    if (sidx[k] != k) identity = false;
  }
  if (n != n_fam) identity = false;
  return Status();
}

void stats_from_counts(const long long* cnt, int64_t m, int64_t n, double* af, double* mac,
                       int64_t* n_valid) {
  for (int64_t j = 0; j < m; ++j) {
    const int64_t alt = cnt[2 * j], miss = cnt[2 * j + 1];
    const int64_t nv = n - miss;
    const double sum = (double)alt;
    af[j] = nv > 0 ? sum / (2.0 * (double)nv) : 0.0;
    const double other = 2.0 * (double)nv - sum;
    mac[j] = sum < other ? sum : other;
    n_valid[j] = nv;
  }
}

// Gather rows of a device-resident .bed into the handle (or count only).
Status bed_gather_dev(const uint8_t* bed_dev, int64_t n_fam, const std::vector<int64_t>& rows,
                             const std::vector<int32_t>& sidx, bool identity, int64_t n,
                             uint32_t* geno_out, int64_t wpr, int64_t* counts_dev,
                             cudaStream_t st) {
  DevBuf d_rows, d_sidx;
  SG_TRY(d_rows.reserve(rows.size() * sizeof(int64_t)));
  SG_CUDA(cudaMemcpyAsync(d_rows.ptr, rows.data(), rows.size() * sizeof(int64_t),
                          cudaMemcpyHostToDevice, st));
  const int32_t* sp = nullptr;
  if (!identity) {
    SG_TRY(d_sidx.reserve(sidx.size() * sizeof(int32_t)));
    SG_CUDA(cudaMemcpyAsync(d_sidx.ptr, sidx.data(), sidx.size() * sizeof(int32_t),
                            cudaMemcpyHostToDevice, st));
    sp = d_sidx.as<int32_t>();
  }
  SG_CUDA(launch_bed_gather(bed_dev, (n_fam + 3) / 4, d_rows.as<int64_t>(), (int64_t)rows.size(),
                            sp, n, geno_out, wpr, counts_dev, st));
  SG_CUDA(cudaStreamSynchronize(st));
  return Status();
}

// ---------------------------------------------------------------------------
// GRM product
// ---------------------------------------------------------------------------
static Status grm_product_fp32(saige_grm* h, const double* v, double* kp, int q,
                               const int32_t* active, cudaStream_t st) {
  SG_TRY(h->v32.reserve((size_t)h->n_pad * sizeof(float)));
  SG_TRY(h->u32.reserve((size_t)h->m_pad * sizeof(float)));
  SG_TRY(h->ypart.reserve((size_t)h->n_splits * h->n_pad * sizeof(float)));
  const float scale = 1.0f / (float)(h->masked ? h->m_active : h->m_eff);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->profiling) {
    SG_CUDA(cudaEventCreate(&e0));
    SG_CUDA(cudaEventCreate(&e1));
    SG_CUDA(cudaEventRecord(e0, st));
  }
  int64_t done = 0;
  for (int c = 0; c < q; ++c) {
    if (active && active[c] != kColActive) continue;
    const double* vc = v + (int64_t)c * h->n_pad;
    double* oc = kp + (int64_t)c * h->n_pad;
    SG_CUDA(launch_to_f32(vc, h->n, h->n_pad, h->v32.as<float>(), st));
    SG_CUDA(launch_fp32_zt(h->geno, h->wpr, h->zlut, h->m_pad, h->v32.as<float>(),
                           h->u32.as<float>(), st));
    if (h->masked) SG_CUDA(mask_rows_f32(h->u32.as<float>(), h->excl.as<uint8_t>(), h->m, st));
    SG_CUDA(launch_fp32_z(h->geno, h->wpr, h->zlut, h->m_pad, h->u32.as<float>(),
                          h->ypart.as<float>(), h->n_splits, st));
    SG_CUDA(launch_fp32_finish(h->ypart.as<float>(), h->n_splits, h->n_pad, h->n, scale, oc, st));
    h->n_kv += 1;
    ++done;
  }
  h->n_kv_launches += 1;
  h->stats.fp32_launches += done;
  if (h->profiling) {
    SG_CUDA(cudaEventRecord(e1, st));
    SG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    h->stats.fp32_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  return Status();
}

Status grm_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                   int precision, cudaStream_t st) {
  if (h->m_eff == 0 || (h->masked && h->m_active == 0)) {
    // pcg.rs:132-134: no markers -> zero vector
    for (int c = 0; c < q; ++c)
      if (!active || active[c] == kColActive)
        SG_CUDA(cudaMemsetAsync(kp + (int64_t)c * h->n_pad, 0, (size_t)h->n_pad * 8, st));
    return Status();
  }
  if (precision == SAIGE_PREC_FP32) return grm_product_fp32(h, v, kp, q, active, st);
  if (precision == SAIGE_PREC_MIXED) return tc_product(h, v, kp, q, active, st);
  return fail(SAIGE_EINVAL, "unknown precision %d", precision);
}

// ---------------------------------------------------------------------------
// PCG driver
// ---------------------------------------------------------------------------
Status pcg_scratch(saige_grm* h, int q, PcgScratch& s) {
  const int64_t ld = h->n_pad;
  const int nb = red_blocks(h->n);
  SG_TRY(h->ws_vec.reserve((size_t)5 * ld * q * sizeof(double)));
  SG_TRY(h->ws_red.reserve((size_t)nb * 3 * q * sizeof(double) + 64));
  SG_TRY(h->ws_cols.reserve((size_t)q * (8 * sizeof(double) + 2 * sizeof(int32_t)) + 256));
  double* base = h->ws_vec.as<double>();
  s.r = base;
  s.z = base + (int64_t)1 * ld * q;
  s.p = base + (int64_t)2 * ld * q;
  s.ap = base + (int64_t)3 * ld * q;
  s.kp = base + (int64_t)4 * ld * q;
  s.partial = h->ws_red.as<double>();
  double* cb = h->ws_cols.as<double>();
  s.cols.rz = cb;
  s.cols.rr = cb + q;
  s.cols.pap = cb + 2 * q;
  s.cols.tol_abs = cb + 3 * q;
  s.small = cb + 4 * q;  // 4q doubles
  int32_t* ib = reinterpret_cast<int32_t*>(cb + 8 * q);
  s.cols.state = ib;
  s.cols.iters = ib + q;
  return Status();
}

Status pcg_run(saige_grm* h, PcgRun& run, cudaStream_t st) {
  const int q = run.q;
  const int64_t n = h->n, ld = h->n_pad;
  PcgScratch s;
  const int ne = run.extra_in && run.extra_out ? run.n_extra : 0;
  SG_TRY(pcg_scratch(h, q + ne, s));  // room for the extra columns in p and kp
  std::vector<int32_t> state((size_t)q, kColActive);
  bool extra_done = ne == 0;
  // With tau1 = 0 the operator is tau0 W^-1 (or tau0 W): tau1 K v contributes only
  // zeros, so no GRM product is formed and K v reads as 0.
  const bool no_k = run.tau1 == 0.0;
  if (no_k) SG_CUDA(cudaMemsetAsync(s.kp, 0, (size_t)ld * q * sizeof(double), st));
  const double* ax0 = run.x0 ? run.ax0 : nullptr;
  if (run.x0 && !run.ax0) {
    // r = b - A x0 (decomposition.rs:225-227)
    SG_CUDA(cudaMemsetAsync(s.cols.state, 0, (size_t)q * sizeof(int32_t), st));
    if (!no_k) SG_TRY(grm_product(h, run.x0, s.kp, q, nullptr, run.precision, st));
    if (run.kx && !no_k)
      SG_CUDA(cudaMemcpyAsync(run.kx, s.kp, (size_t)ld * q * sizeof(double),
                              cudaMemcpyDeviceToDevice, st));
    if (run.w_inverse)
      SG_CUDA(pcg_apply(run.x0, s.kp, run.wv, run.tau0, run.tau1, s.ap, n, ld, q, s.cols,
                        s.partial, st));
    else
      SG_CUDA(pcg_apply_w(run.x0, s.kp, run.wv, run.tau0, run.tau1, s.ap, n, ld, q, s.cols,
                          s.partial, st));
    ax0 = s.ap;
  }
  if (run.kx && !(run.x0 && !run.ax0)) {
    if (run.x0 && run.kx0)
      SG_CUDA(cudaMemcpyAsync(run.kx, run.kx0, (size_t)ld * q * sizeof(double),
                              cudaMemcpyDeviceToDevice, st));
    else
      SG_CUDA(cudaMemsetAsync(run.kx, 0, (size_t)ld * q * sizeof(double), st));
  }
  run.kx_valid = run.kx && !no_k && (!run.x0 || !run.ax0 || run.kx0);
  SG_CUDA(pcg_start(run.b, run.x0, ax0, run.d, run.x, s.r, s.z, s.p, n, ld, q, run.tol,
                    run.force_step && run.x0 != nullptr, s.cols, s.partial, s.small, st));
  if (run.max_iter <= 0) {
    // the loop body never runs; converged is the initial test
    SG_CUDA(cudaMemcpyAsync(state.data(), s.cols.state, (size_t)q * 4, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
  } else {
    for (;;) {
      SG_CUDA(cudaMemcpyAsync(state.data(), s.cols.state, (size_t)q * 4, cudaMemcpyDeviceToHost,
                              st));
      SG_CUDA(cudaStreamSynchronize(st));
      bool any = false;
      for (int c = 0; c < q; ++c) any |= state[(size_t)c] == kColActive;
      if (!any) break;
      if (!no_k && !extra_done) {
        // the extra columns ride in this launch
        SG_CUDA(cudaMemcpyAsync(s.p + (size_t)q * ld, run.extra_in, (size_t)ld * ne * sizeof(double),
                                cudaMemcpyDeviceToDevice, st));
        std::vector<int32_t> st2 = state;
        st2.resize((size_t)(q + ne), kColActive);
        SG_TRY(grm_product(h, s.p, s.kp, q + ne, st2.data(), run.precision, st));
        SG_CUDA(cudaMemcpyAsync(run.extra_out, s.kp + (size_t)q * ld, (size_t)ld * ne * sizeof(double),
                                cudaMemcpyDeviceToDevice, st));
        extra_done = true;
      } else if (!no_k) {
        SG_TRY(grm_product(h, s.p, s.kp, q, state.data(), run.precision, st));
      }
      if (!no_k && run.keep_p && run.keep_kp)
        for (int c = 0; c < std::min(run.keep_cols, q) && run.kept < run.keep_cap; ++c) {
          if (state[(size_t)c] != kColActive) continue;
          SG_CUDA(cudaMemcpyAsync(run.keep_p + (size_t)run.kept * ld, s.p + (size_t)c * ld,
                                  (size_t)ld * 8, cudaMemcpyDeviceToDevice, st));
          SG_CUDA(cudaMemcpyAsync(run.keep_kp + (size_t)run.kept * ld, s.kp + (size_t)c * ld,
                                  (size_t)ld * 8, cudaMemcpyDeviceToDevice, st));
          ++run.kept;
        }
      if (run.w_inverse)
        SG_CUDA(pcg_apply(s.p, s.kp, run.wv, run.tau0, run.tau1, s.ap, n, ld, q, s.cols,
                          s.partial, st));
      else
        SG_CUDA(pcg_apply_w(s.p, s.kp, run.wv, run.tau0, run.tau1, s.ap, n, ld, q, s.cols,
                            s.partial, st));
      SG_CUDA(pcg_step(run.x, s.r, s.z, s.p, s.ap, run.d, n, ld, q, run.max_iter, s.cols,
                       s.partial, s.small, st, run.kx_valid ? run.kx : nullptr, s.kp));
    }
  }
  if (!extra_done)
    SG_TRY(grm_product(h, run.extra_in, run.extra_out, ne, nullptr, run.precision, st));
  if (run.r_out)
    SG_CUDA(cudaMemcpyAsync(run.r_out, s.r, (size_t)ld * q * sizeof(double),
                            cudaMemcpyDeviceToDevice, st));
  std::vector<double> rr((size_t)q);
  run.iters.assign((size_t)q, 0);
  run.state = state;
  SG_CUDA(cudaMemcpyAsync(run.iters.data(), s.cols.iters, (size_t)q * 4, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaMemcpyAsync(rr.data(), s.cols.rr, (size_t)q * 8, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  run.resid.resize((size_t)q);
  run.total_iters = 0;
  for (int c = 0; c < q; ++c) {
    run.resid[(size_t)c] = sqrt(rr[(size_t)c]);
    if (run.max_iter <= 0 && state[(size_t)c] == kColActive) run.state[(size_t)c] = kColMaxIter;
    run.total_iters += run.iters[(size_t)c];
  }
  return Status();
}

}  // namespace saige

using namespace saige;

// ===========================================================================
// C ABI
// ===========================================================================
#define SG_API extern "C" __attribute__((visibility("default")))

#define SG_GUARD_BEGIN try {
#define SG_GUARD_END                                                          \
  }                                                                           \
  catch (const std::bad_alloc&) {                                             \
    return fail(SAIGE_ENOMEM, "host allocation failed").code;                 \
  }                                                                           \
  catch (...) {                                                               \
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;               \
  }

SG_API const char* saige_last_error(void) { return last_error(); }

SG_API int32_t saige_version(void) { return 1 * 10000 + 0 * 100 + 0; }

SG_API int32_t saige_device_count(void) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  int usable = 0;
  for (int d = 0; d < count; ++d) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10 && p.minor == 0) ++usable;
  }
  return usable;
}

static int32_t marker_stats_impl(const uint8_t* bed, bool on_device, size_t bed_len,
                                 int64_t n_fam, int64_t m_tot, const int64_t* sample_idx,
                                 int64_t n, double* af, double* mac, int64_t* n_valid) {
  if (!bed || !af || !mac || !n_valid || m_tot < 0) return fail(SAIGE_EINVAL, "null argument").code;
  uint8_t hdr[3] = {0, 0, 0};
  Status s;
  cudaStream_t st = nullptr;
  // a host .bed is checked before any device call (errors need no GPU)
  if (!on_device) {
    if (bed_len >= 3) memcpy(hdr, bed, 3);
  } else {
    s = pick_device(-1, nullptr);
    if (!s.ok()) return s.code;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      return fail(SAIGE_ECUDA, "stream creation failed").code;
    // on this call's own stream: a legacy-stream copy would wait for other work
    if (bed_len >= 3 && (cudaMemcpyAsync(hdr, bed, 3, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                         cudaStreamSynchronize(st) != cudaSuccess)) {
      cudaStreamDestroy(st);
      return fail(SAIGE_ECUDA, "reading the bed header from device memory failed").code;
    }
  }
  s = check_bed_header(hdr, bed_len, n_fam, m_tot);
  std::vector<int32_t> sidx;
  bool identity = true;
  if (s.ok()) s = check_subset(sample_idx, n, n_fam, sidx, identity);
  if (s.ok() && !st) {
    s = pick_device(-1, nullptr);
    if (s.ok() && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
      s = fail(SAIGE_ECUDA, "stream creation failed");
  }
  if (!s.ok()) {
    if (st) cudaStreamDestroy(st);
    return s.code;
  }
  const int64_t bpm = (n_fam + 3) / 4;
  const size_t used = (size_t)(3 + bpm * m_tot);
  // every buffer below is used on st only: its release waits for st, not the device
  ReleaseScope rs(ReleaseMode::kStream, st);
  DevBuf d_bed, d_cnt;
  auto body = [&]() -> Status {
    SG_TRY(d_cnt.reserve((size_t)std::max<int64_t>(m_tot, 1) * 2 * sizeof(int64_t)));
    const uint8_t* src = bed;
    if (!on_device) {
      SG_TRY(d_bed.reserve(used));
      SG_CUDA(cudaMemcpyAsync(d_bed.ptr, bed, used, cudaMemcpyHostToDevice, st));
      src = d_bed.as<uint8_t>();
    }
    std::vector<int64_t> rows((size_t)m_tot);
    for (int64_t j = 0; j < m_tot; ++j) rows[(size_t)j] = j;
    if (m_tot > 0)
      SG_TRY(bed_gather_dev(src, n_fam, rows, sidx, identity, n, nullptr, 0, d_cnt.as<int64_t>(),
                            st));
    std::vector<int64_t> cnt((size_t)m_tot * 2);
    if (m_tot > 0) {
      SG_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt.ptr, cnt.size() * 8, cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaStreamSynchronize(st));
    }
    stats_from_counts(reinterpret_cast<const long long*>(cnt.data()), m_tot, n, af, mac, n_valid);
    return Status();
  };
  s = body();
  d_bed.release();
  d_cnt.release();
  cudaStreamDestroy(st);
  return s.code;
}

SG_API int32_t saige_bed_marker_stats(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                      int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                      double* af, double* mac, int64_t* n_valid) {
  SG_GUARD_BEGIN
  set_error("");
  return marker_stats_impl(bed, false, bed_len, n_fam, m_tot, sample_idx, n, af, mac, n_valid);
  SG_GUARD_END
}

SG_API int32_t saige_bed_marker_stats_dev(const uint8_t* bed_dev, size_t bed_len, int64_t n_fam,
                                          int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                          double* af, double* mac, int64_t* n_valid) {
  SG_GUARD_BEGIN
  set_error("");
  return marker_stats_impl(bed_dev, true, bed_len, n_fam, m_tot, sample_idx, n, af, mac, n_valid);
  SG_GUARD_END
}

SG_API int32_t saige_grm_set_profiling(saige_grm* h, int32_t on) {
  if (!h) return fail(SAIGE_EINVAL, "null handle").code;
  std::lock_guard<std::recursive_mutex> lk(h->mu);
  h->profiling = on != 0;
  return SAIGE_OK;
}

SG_API int32_t saige_grm_get_stats(const saige_grm* h, saige_grm_stats* out) {
  if (!h || !out) return fail(SAIGE_EINVAL, "null argument").code;
  *out = h->stats;
  out->n_kv = h->n_kv;
  out->n_kv_launches = h->n_kv_launches;
  out->missing_listed = tc_missing_listed(h);
  return SAIGE_OK;
}

SG_API int32_t saige_grm_reset_stats(saige_grm* h) {
  if (!h) return fail(SAIGE_EINVAL, "null handle").code;
  std::lock_guard<std::recursive_mutex> lk(h->mu);
  h->stats = saige_grm_stats{};
  h->n_kv = 0;
  h->n_kv_launches = 0;
  return SAIGE_OK;
}

SG_API int64_t saige_kernel_launches(void) { return launches_total(); }

SG_API int64_t saige_tc_autotune_trials(void) { return tc_autotune_trials(); }

SG_API int32_t saige_tc_set_wait_budget(int64_t cycles) {
  tc_set_wait_budget((long long)cycles);
  return SAIGE_OK;
}

SG_API int32_t saige_release_cached_memory(void) {
  SG_GUARD_BEGIN
  release_cached_blocks();
  return SAIGE_OK;
  SG_GUARD_END
}

SG_API int32_t saige_rademacher_probes(uint64_t seed, int32_t n_vec, int64_t n, double* out,
                                      int32_t device) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out || n_vec <= 0 || n <= 0) return fail(SAIGE_EINVAL, "null argument or empty size").code;
  int dev = 0;
  Status ps = pick_device(device, &dev);
  if (!ps.ok()) return ps.code;
  auto body = [&]() -> Status {
    DevBuf d;
    SG_TRY(d.reserve((size_t)n_vec * n * sizeof(double)));
    const ChaCha8 rng(seed);
    SG_CUDA(rademacher_probes_dev(rng.key(), d.as<double>(), n, n, n_vec, 0));
    SG_CUDA(cudaMemcpy(out, d.ptr, (size_t)n_vec * n * sizeof(double), cudaMemcpyDeviceToHost));
    return Status();
  };
  return body().code;
  SG_GUARD_END
}

// fit_null.rs:209-222: the QC a marker passes to enter the GRM or the variance-ratio
// candidates.
static bool qc_pass(double af, int64_t n_valid, int64_t n, double min_maf, double max_missing) {
  const double missing_rate = 1.0 - ((double)n_valid / (double)n);
  return af >= min_maf && af <= 1.0 - min_maf && missing_rate <= max_missing;
}

// fit_null.rs:234-243: 1000 draws of gen_range(0..pass.len()) from ChaCha8(seed),
// sorted and deduplicated; a drawn marker with mac >= 20 is a variance-ratio
// candidate (flags[i] = 1 for position i of pass), every other passing marker is a
// GRM marker.
static void vr_candidate_flags(const std::vector<int64_t>& pass, const double* mac, uint64_t seed,
                               std::vector<uint8_t>& flags) {
  ChaCha8 rng(seed);
  std::vector<uint64_t> cand(1000);
  for (auto& c : cand) c = rng.gen_range(0, (uint64_t)pass.size());
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  flags.assign(pass.size(), 0);
  for (uint64_t c : cand)
    if (mac[pass[(size_t)c]] >= 20.0) flags[(size_t)c] = 1;
}

SG_API int32_t saige_select_grm_markers(const double* af, const double* mac,
                                        const int64_t* n_valid, int64_t m_tot, int64_t n,
                                        double min_maf, double max_missing, uint64_t seed,
                                        int64_t* grm_idx, int64_t* m_grm, int64_t* vr_idx,
                                        int64_t* m_vr) {
  SG_GUARD_BEGIN
  set_error("");
  if (!af || !mac || !n_valid || !grm_idx || !m_grm || !vr_idx || !m_vr || n <= 0)
    return fail(SAIGE_EINVAL, "null argument or n <= 0").code;
  // fit_null.rs:209-222
  std::vector<int64_t> pass;
  pass.reserve((size_t)m_tot);
  for (int64_t j = 0; j < m_tot; ++j)
    if (qc_pass(af[j], n_valid[j], n, min_maf, max_missing)) pass.push_back(j);
  *m_grm = 0;
  *m_vr = 0;
  if (pass.empty())
    return fail(SAIGE_EINVAL, "no marker passes QC (gen_range(0..0) in the reference)").code;
  std::vector<uint8_t> vr;
  vr_candidate_flags(pass, mac, seed, vr);
  int64_t g = 0, v = 0;
  for (size_t i = 0; i < pass.size(); ++i) {
    if (vr[i]) vr_idx[v++] = pass[i];
    else grm_idx[g++] = pass[i];
  }
  *m_grm = g;
  *m_vr = v;
  return SAIGE_OK;
  SG_GUARD_END
}

static int32_t create_from_bed_impl(const uint8_t* bed, bool on_device, size_t bed_len,
                                    int64_t n_fam, int64_t m_tot, const int64_t* sample_idx,
                                    int64_t n, const int64_t* marker_idx, int64_t m,
                                    const double* allele_freqs, int32_t device, saige_grm** out) {
  if (!bed || !out || (m > 0 && (!marker_idx || !allele_freqs)) || m < 0)
    return fail(SAIGE_EINVAL, "null argument").code;
  *out = nullptr;
  std::vector<uint8_t> hdr(3, 0);
  int dev;
  Status s = pick_device(device, &dev);
  if (!s.ok()) return s.code;
  if (on_device) {
    if (bed_len >= 3) {
      // on a stream of this call: a legacy-stream copy would wait for other work
      cudaStream_t hs;
      if (cudaStreamCreateWithFlags(&hs, cudaStreamNonBlocking) != cudaSuccess)
        return fail(SAIGE_ECUDA, "stream creation failed").code;
      const bool ok = cudaMemcpyAsync(hdr.data(), bed, 3, cudaMemcpyDeviceToHost, hs) == cudaSuccess &&
                      cudaStreamSynchronize(hs) == cudaSuccess;
      cudaStreamDestroy(hs);
      if (!ok) return fail(SAIGE_ECUDA, "reading the bed header from device memory failed").code;
    }
  } else if (bed_len >= 3) {
    memcpy(hdr.data(), bed, 3);
  }
  s = check_bed_header(hdr.data(), bed_len, n_fam, m_tot);
  if (!s.ok()) return s.code;
  std::vector<int32_t> sidx;
  bool identity;
  s = check_subset(sample_idx, n, n_fam, sidx, identity);
  if (!s.ok()) return s.code;
  std::vector<int64_t> rows((size_t)m);
  for (int64_t r = 0; r < m; ++r) {
    if (marker_idx[r] < 0 || marker_idx[r] >= m_tot)
      return fail(SAIGE_EINVAL, "marker_idx[%lld] out of range", (long long)r).code;
    rows[(size_t)r] = marker_idx[r];
  }
  saige_grm* h = new saige_grm();
  h->device = dev;
  PhaseTimer tm;
  auto body = [&]() -> Status {
    SG_TRY(grm_alloc(h, n, m));  // creates the handle's stream
    // the gather's temporaries are used on the handle's stream only
    ReleaseScope rs(ReleaseMode::kStream, h->stream);
    tm.mark(" grm alloc");
    SG_TRY(grm_upload_meta(h, allele_freqs));
    tm.mark(" grm meta");
    if (m > 0) {
      const int64_t bpm = (n_fam + 3) / 4;
      const size_t used = (size_t)(3 + bpm * m_tot);
      DevBuf d_bed;
      const uint8_t* src = bed;
      if (!on_device) {
        SG_TRY(d_bed.reserve(used));
        SG_CUDA(cudaMemcpyAsync(d_bed.ptr, bed, used, cudaMemcpyHostToDevice, h->stream));
        src = d_bed.as<uint8_t>();
      }
      SG_TRY(bed_gather_dev(src, n_fam, rows, sidx, identity, n, h->geno, h->wpr, nullptr,
                            h->stream));
      tm.mark(" grm gather");
      SG_TRY(grm_blank_degenerate_rows(h, allele_freqs));
      tm.mark(" grm blank");
    }
    SG_CUDA(cudaStreamSynchronize(h->stream));
    return Status();
  };
  s = body();
  if (!s.ok()) {
    grm_free(h);
    return s.code;
  }
  *out = h;
  return SAIGE_OK;
}

namespace saige {

Status grm_stream_rows_finish(saige_grm* h, const std::vector<int64_t>& pass, const double* af,
                              const double* mac, uint64_t seed, std::vector<int64_t>& vidx) {
  if (pass.empty())
    return fail(SAIGE_EINVAL, "no marker passes QC (gen_range(0..0) in the reference)");
  std::vector<uint8_t> flags;
  vr_candidate_flags(pass, mac, seed, flags);
  const int64_t rows = (int64_t)pass.size();
  h->m = rows;
  h->m_pad = round_up(rows, kMarkerPad);
  // padding rows: all codes 11, 2p = 1/s = 0
  SG_CUDA(cudaMemsetAsync(h->geno + (size_t)rows * h->wpr, 0xFF,
                          (size_t)(h->m_pad - rows) * h->wpr * 4, h->stream));
  std::vector<double> row_af((size_t)rows);
  for (int64_t r = 0; r < rows; ++r) row_af[(size_t)r] = af[(size_t)pass[(size_t)r]];
  std::vector<float4> zl;
  std::vector<double> tp, is;
  marker_meta(row_af.data(), rows, h->m_pad, zl, tp, is);
  vidx.clear();
  for (int64_t r = 0; r < rows; ++r) {
    if (!flags[(size_t)r]) continue;
    vidx.push_back(pass[(size_t)r]);
    zl[(size_t)r] = make_float4(0.f, 0.f, 0.f, 0.f);
    tp[(size_t)r] = 0.0;
    is[(size_t)r] = 0.0;
  }
  SG_CUDA(cudaMemcpyAsync(h->zlut, zl.data(), zl.size() * sizeof(float4), cudaMemcpyHostToDevice,
                          h->stream));
  SG_CUDA(cudaMemcpyAsync(h->two_p, tp.data(), tp.size() * 8, cudaMemcpyHostToDevice, h->stream));
  SG_CUDA(cudaMemcpyAsync(h->inv_s, is.data(), is.size() * 8, cudaMemcpyHostToDevice, h->stream));
  h->m_eff = rows - (int64_t)vidx.size();
  h->n_splits = fp32_z_splits(h->n_pad, h->m_pad);
  SG_CUDA(cudaStreamSynchronize(h->stream));  // the host vectors go out of scope
  return Status();
}

}  // namespace saige

// The fit-null GRM built while the .bed streams in from pinned host memory.  The
// upload runs in marker chunks on a copy stream; as each chunk lands, the handle's
// stream counts its alleles and missing calls (K1), the host applies the marker QC
// to the chunk, and the chunk's passing markers are gathered into the next rows of
// the handle and tiled as soon as a 128-row group is complete — all under the
// transfer of the chunks that follow.  The rows are every QC-passing marker in .bed
// order; the variance-ratio candidates, drawn only once the number of passing
// markers is known, stay in place with 2p = 1/s = 0 (so that every product gets an
// exact zero from them) and m_eff = m - candidates is the GRM's M.  The integer
// products of the MIXED path are then bit-identical to those of a handle holding
// only the GRM markers; FP32 products would sum in another grouping, so this build
// serves MIXED fits only.
namespace saige {

Status stream_fit_null_grm(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                           const int64_t* sample_idx, int64_t n, double min_maf,
                           double max_missing, uint64_t seed, DevBuf& d_bed,
                           std::vector<double>& af, std::vector<double>& mac,
                           std::vector<int64_t>& nv, std::vector<int64_t>& vidx, int64_t& m_grm,
                           saige_grm** out) {
  *out = nullptr;
  SG_TRY(check_bed_header(bed, bed_len, n_fam, m_tot));
  std::vector<int32_t> sidx;
  bool identity = true;
  SG_TRY(check_subset(sample_idx, n, n_fam, sidx, identity));
  if (d_bed.bytes < bed_len) return fail(SAIGE_EINVAL, "device .bed buffer too small");
  int dev = 0;
  SG_TRY(pick_device(-1, &dev));
  const int64_t bpm = (n_fam + 3) / 4;
  const int64_t cap = round_up(m_tot, kMarkerPad);
  saige_grm* h = new saige_grm();
  h->device = dev;
  struct Streams {
    cudaStream_t c = nullptr;
    std::vector<cudaEvent_t> ev;
    cudaStream_t k = nullptr;
    ~Streams() {
      if (c) cudaStreamSynchronize(c);
      if (k) cudaStreamSynchronize(k);
      for (cudaEvent_t e : ev) cudaEventDestroy(e);
      if (c) cudaStreamDestroy(c);
    }
  };
  // Host-mapped memory for what crosses PCIe beside the .bed (row lists, counts): no
  // copy of it queues behind the chunks on the copy engines.  One block is kept for
  // the process and reused (pinning and unpinning host memory on every call cost
  // milliseconds, once close to a second); a call that finds it in use by another
  // thread takes a block of its own.
  struct Mapped {
    void* p = nullptr;
    bool own = false;
    ~Mapped() {
      if (own) {
        cudaFreeHost(p);
      } else if (p) {
        std::lock_guard<std::mutex> lk(g_mapped_mu);
        g_mapped_busy = false;
      }
    }
    Status take(size_t bytes) {
      {
        std::lock_guard<std::mutex> lk(g_mapped_mu);
        if (!g_mapped_busy) {
          if (g_mapped_bytes < bytes) {
            if (g_mapped) cudaFreeHost(g_mapped);
            g_mapped = nullptr;
            g_mapped_bytes = 0;
            SG_CUDA(cudaHostAlloc(&g_mapped, bytes, cudaHostAllocMapped));
            g_mapped_bytes = bytes;
          }
          g_mapped_busy = true;
          p = g_mapped;
          return Status();
        }
      }
      own = true;
      SG_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocMapped));
      return Status();
    }
  };
  PhaseTimer tm;
  auto body = [&]() -> Status {
    Mapped mp;  // outlives the streams' last use of it (destroyed after ss)
    Streams ss;
    SG_CUDA(cudaStreamCreateWithFlags(&ss.c, cudaStreamNonBlocking));
    // the sample subset ahead of the .bed on the copy stream (the counts need it)
    DevBuf d_sidx;
    const int32_t* sp = nullptr;
    if (!identity) {
      SG_TRY(d_sidx.reserve(sidx.size() * 4));
      SG_CUDA(cudaMemcpyAsync(d_sidx.ptr, sidx.data(), sidx.size() * 4, cudaMemcpyHostToDevice,
                              ss.c));
      sp = d_sidx.as<int32_t>();
    }
    // every chunk's copy is queued first, so that all the set-up below overlaps the
    // transfer; the kernels follow chunk by chunk
    constexpr int kChunks = 32;
    const int64_t per = ceil_div(m_tot, (int64_t)kChunks);
    uint8_t* dst = d_bed.as<uint8_t>();
    for (int64_t j0 = 0; j0 < m_tot; j0 += per) {
      const int64_t j1 = std::min(m_tot, j0 + per);
      const size_t lo = j0 == 0 ? 0 : (size_t)(3 + j0 * bpm);
      const size_t hi = j1 == m_tot ? bed_len : (size_t)(3 + j1 * bpm);
      SG_CUDA(cudaMemcpyAsync(dst + lo, bed + lo, hi - lo, cudaMemcpyHostToDevice, ss.c));
      cudaEvent_t e = nullptr;
      SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      ss.ev.push_back(e);
      SG_CUDA(cudaEventRecord(e, ss.c));
    }
    h->n = n;
    h->n_pad = round_up(std::max<int64_t>(n, 1), kSamplePad);
    h->wpr = h->n_pad / 16;
    SG_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    ss.k = h->stream;
    SG_TRY(h->geno_buf.reserve((size_t)cap * h->wpr * 4));
    h->geno = h->geno_buf.as<uint32_t>();
    SG_TRY(grm_alloc_meta(h, cap));
    SG_TRY(tc_stream_begin(h, cap));
    // all[j] = j (the rows the counts read), prow (the passing rows, in .bed order),
    // cnt (alt and missing counts per marker)
    SG_TRY(mp.take((size_t)m_tot * 32));
    int64_t* all_h = static_cast<int64_t*>(mp.p);
    int64_t* prow_h = all_h + m_tot;
    int64_t* cnt_h = prow_h + m_tot;
    void* mapped_dev = nullptr;
    SG_CUDA(cudaHostGetDevicePointer(&mapped_dev, mp.p, 0));
    const int64_t* all_d = static_cast<const int64_t*>(mapped_dev);
    const int64_t* prow_d = all_d + m_tot;
    int64_t* cnt_d = const_cast<int64_t*>(prow_d) + m_tot;
    for (int64_t j = 0; j < m_tot; ++j) all_h[j] = j;
    cudaEvent_t counted = nullptr;
    SG_CUDA(cudaEventCreateWithFlags(&counted, cudaEventDisableTiming));
    ss.ev.push_back(counted);
    std::vector<int64_t> pass;
    pass.reserve((size_t)m_tot);
    int64_t mt_done = 0;
    size_t chunk = 0;
    for (int64_t j0 = 0; j0 < m_tot; j0 += per, ++chunk) {
      const int64_t j1 = std::min(m_tot, j0 + per);
      SG_CUDA(cudaStreamWaitEvent(h->stream, ss.ev[chunk], 0));
      SG_CUDA(launch_bed_gather(dst, bpm, all_d + j0, j1 - j0, sp, n, nullptr, 0, cnt_d + 2 * j0,
                                h->stream));
      SG_CUDA(cudaEventRecord(counted, h->stream));
      SG_CUDA(cudaEventSynchronize(counted));
      const size_t p0 = pass.size();
      std::vector<int64_t> degenerate;
      for (int64_t j = j0; j < j1; ++j) {
        const int64_t alt = cnt_h[2 * j], miss = cnt_h[2 * j + 1];
        const int64_t valid = n - miss;
        // traits.rs:42-54, the same f64 operations on the same exact integers
        const double sum = (double)alt;
        af[(size_t)j] = valid > 0 ? sum / (2.0 * (double)valid) : 0.0;
        const double other = 2.0 * (double)valid - sum;
        mac[(size_t)j] = sum < other ? sum : other;
        nv[(size_t)j] = valid;
        if (!qc_pass(af[(size_t)j], valid, n, min_maf, max_missing)) continue;
        const double p = af[(size_t)j];
        if (!(sqrt(2.0 * p * (1.0 - p)) > 1e-10)) degenerate.push_back((int64_t)pass.size());
        prow_h[pass.size()] = j;
        pass.push_back(j);
      }
      const size_t p1 = pass.size();
      if (p1 > p0) {
        SG_CUDA(launch_bed_gather(dst, bpm, prow_d + p0, (int64_t)(p1 - p0), sp, n,
                                  h->geno + p0 * (size_t)h->wpr, h->wpr, nullptr, h->stream));
        // a zero standardised column: codes 11, as grm_blank_degenerate_rows does
        for (int64_t r : degenerate)
          SG_CUDA(cudaMemsetAsync(h->geno + (size_t)r * h->wpr, 0xFF, (size_t)h->wpr * 4,
                                  h->stream));
      }
      const int64_t mt_full = (int64_t)p1 / kMarkerPad;
      SG_TRY(tc_stream_tiles(h, mt_done, mt_full, h->stream));
      mt_done = mt_full;
    }
    tm.mark(" stream chunks");
    SG_TRY(grm_stream_rows_finish(h, pass, af.data(), mac.data(), seed, vidx));
    SG_TRY(tc_stream_tiles(h, mt_done, h->m_pad / kMarkerPad, h->stream));
    m_grm = h->m_eff;
    SG_CUDA(cudaStreamSynchronize(h->stream));
    SG_CUDA(cudaStreamSynchronize(ss.c));
    tm.mark(" stream tail");
    return Status();
  };
  Status s = body();
  tm.mark(" stream exit");
  if (!s.ok()) {
    grm_free(h);
    return s;
  }
  *out = h;
  return Status();
}

}  // namespace saige

SG_API int32_t saige_grm_create_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                         int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                         const int64_t* marker_idx, int64_t m,
                                         const double* allele_freqs, int32_t device,
                                         saige_grm** out) {
  SG_GUARD_BEGIN
  set_error("");
  return create_from_bed_impl(bed, false, bed_len, n_fam, m_tot, sample_idx, n, marker_idx, m,
                              allele_freqs, device, out);
  SG_GUARD_END
}

namespace saige {

Status grm_shell_create(int dev, int64_t n, int64_t m, const double* af, saige_grm** out) {
  *out = nullptr;
  saige_grm* h = new saige_grm();
  h->device = dev;
  Status s = grm_alloc(h, n, m);
  if (s.ok() && m > 0) s = grm_upload_meta(h, af);
  if (!s.ok()) {
    grm_free(h);
    return s;
  }
  *out = h;
  return Status();
}

Status grm_shell_finish(saige_grm* h, const double* af) {
  if (h->m > 0) SG_TRY(grm_blank_degenerate_rows(h, af));
  SG_CUDA(cudaStreamSynchronize(h->stream));
  return Status();
}

void grm_shell_destroy(saige_grm* h) { grm_free(h); }

Status grm_shell_create_cap(int dev, int64_t n, int64_t rows_cap, saige_grm** out) {
  *out = nullptr;
  saige_grm* h = new saige_grm();
  h->device = dev;
  Status s = grm_alloc(h, n, rows_cap);
  if (!s.ok()) {
    grm_free(h);
    return s;
  }
  *out = h;
  return Status();
}

bool marker_qc_pass(double af, int64_t n_valid, int64_t n, double min_maf, double max_missing) {
  return qc_pass(af, n_valid, n, min_maf, max_missing);
}

}  // namespace saige

SG_API int32_t saige_grm_create_from_bed_dev(const uint8_t* bed_dev, size_t bed_len,
                                             int64_t n_fam, int64_t m_tot,
                                             const int64_t* sample_idx, int64_t n,
                                             const int64_t* marker_idx, int64_t m,
                                             const double* allele_freqs, int32_t device,
                                             saige_grm** out) {
  SG_GUARD_BEGIN
  set_error("");
  return create_from_bed_impl(bed_dev, true, bed_len, n_fam, m_tot, sample_idx, n, marker_idx, m,
                              allele_freqs, device, out);
  SG_GUARD_END
}

SG_API int32_t saige_grm_create_from_dosages(const double* dosages, int64_t n, int64_t m,
                                             const double* allele_freqs, int32_t device,
                                             saige_grm** out) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out || n <= 0 || m < 0 || (m > 0 && (!dosages || !allele_freqs)))
    return fail(SAIGE_EINVAL, "null argument or bad dimension").code;
  // Encode hard calls as a .bed image and reuse the packed path.
  const int64_t bpm = (n + 3) / 4;
  std::vector<uint8_t> bed((size_t)(3 + bpm * m), 0);
  bed[0] = 0x6C;
  bed[1] = 0x1B;
  bed[2] = 0x01;
  for (int64_t j = 0; j < m; ++j) {
    uint8_t* row = bed.data() + 3 + j * bpm;
    for (int64_t i = 0; i < n; ++i) {
      const double g = dosages[j * n + i];
      uint32_t code;
      if (isnan(g)) code = 1;
      else if (g == 2.0) code = 0;
      else if (g == 1.0) code = 2;
      else if (g == 0.0) code = 3;
      else
        return fail(SAIGE_EINVAL, "dosage[%lld][%lld] = %g is not a hard call (0, 1, 2 or NaN)",
                    (long long)j, (long long)i, g)
            .code;
      row[i >> 2] |= (uint8_t)(code << ((i & 3) * 2));
    }
  }
  std::vector<int64_t> rows((size_t)m);
  for (int64_t j = 0; j < m; ++j) rows[(size_t)j] = j;
  return create_from_bed_impl(bed.data(), false, bed.size(), n, m, nullptr, n, rows.data(), m,
                              allele_freqs, device, out);
  SG_GUARD_END
}

SG_API int32_t saige_grm_destroy(saige_grm* h) {
  SG_GUARD_BEGIN
  grm_free(h);
  return SAIGE_OK;
  SG_GUARD_END
}

SG_API int32_t saige_grm_dims(const saige_grm* h, int64_t* n, int64_t* m) {
  if (!h) return fail(SAIGE_EINVAL, "null handle").code;
  if (n) *n = h->n;
  if (m) *m = h->m;
  return SAIGE_OK;
}

// Copy a host block (n x q, vector-major) into a padded device block.
static Status upload_block(saige_grm* h, const double* src, double* dst, int q, cudaStream_t st) {
  SG_CUDA(cudaMemcpy2DAsync(dst, (size_t)h->n_pad * 8, src, (size_t)h->n * 8, (size_t)h->n * 8, q,
                            cudaMemcpyHostToDevice, st));
  SG_CUDA(zero_pad(dst, h->n, h->n_pad, q, st));
  return Status();
}
static Status download_block(saige_grm* h, const double* src, double* dst, int q, cudaStream_t st) {
  SG_CUDA(cudaMemcpy2DAsync(dst, (size_t)h->n * 8, src, (size_t)h->n_pad * 8, (size_t)h->n * 8, q,
                            cudaMemcpyDeviceToHost, st));
  return Status();
}
static Status devcopy_block(saige_grm* h, const double* src, int64_t sld, double* dst, int64_t dld,
                            int q, cudaStream_t st) {
  SG_CUDA(cudaMemcpy2DAsync(dst, (size_t)dld * 8, src, (size_t)sld * 8, (size_t)h->n * 8, q,
                            cudaMemcpyDeviceToDevice, st));
  return Status();
}

SG_API int32_t saige_grm_matvec(saige_grm* h, const double* v, double* out, int64_t n,
                                int32_t nrhs, int32_t precision) {
  SG_GUARD_BEGIN
  set_error("");
  if (!h || !v || !out) return fail(SAIGE_EINVAL, "null argument").code;
  if (n != h->n) return fail(SAIGE_EINVAL, "v.len() = %lld != n_samples = %lld", (long long)n,
                             (long long)h->n).code;  // pcg.rs:129
  if (nrhs <= 0) return fail(SAIGE_EINVAL, "nrhs must be positive").code;
  std::lock_guard<std::recursive_mutex> lk(h->mu);
  DeviceGuard dg(h->device);
  auto body = [&]() -> Status {
    const size_t blk = (size_t)h->n_pad * nrhs * sizeof(double);
    SG_TRY(h->ws_io.reserve(2 * blk));
    double* dv = h->ws_io.as<double>();
    double* dk = dv + (size_t)h->n_pad * nrhs;
    SG_TRY(upload_block(h, v, dv, nrhs, h->stream));
    SG_TRY(grm_product(h, dv, dk, nrhs, nullptr, precision, h->stream));
    SG_TRY(download_block(h, dk, out, nrhs, h->stream));
    SG_CUDA(cudaStreamSynchronize(h->stream));
    return Status();
  };
  return body().code;
  SG_GUARD_END
}

SG_API int32_t saige_grm_matvec_dev(saige_grm* h, const double* v_dev, double* out_dev, int64_t n,
                                    int32_t nrhs, int32_t precision, void* stream) {
  SG_GUARD_BEGIN
  set_error("");
  if (!h || !v_dev || !out_dev) return fail(SAIGE_EINVAL, "null argument").code;
  if (n != h->n) return fail(SAIGE_EINVAL, "n mismatch").code;
  if (nrhs <= 0) return fail(SAIGE_EINVAL, "nrhs must be positive").code;
  std::lock_guard<std::recursive_mutex> lk(h->mu);
  DeviceGuard dg(h->device);
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  auto body = [&]() -> Status {
    const size_t blk = (size_t)h->n_pad * nrhs * sizeof(double);
    SG_TRY(h->ws_io.reserve(2 * blk));
    double* dv = h->ws_io.as<double>();
    double* dk = dv + (size_t)h->n_pad * nrhs;
    SG_TRY(devcopy_block(h, v_dev, h->n, dv, h->n_pad, nrhs, st));
    SG_CUDA(zero_pad(dv, h->n, h->n_pad, nrhs, st));
    SG_TRY(grm_product(h, dv, dk, nrhs, nullptr, precision, st));
    SG_TRY(devcopy_block(h, dk, h->n_pad, out_dev, h->n, nrhs, st));
    SG_CUDA(cudaStreamSynchronize(st));
    return Status();
  };
  return body().code;
  SG_GUARD_END
}

SG_API int32_t saige_grm_diag(saige_grm* h, double* out, int64_t n) {
  SG_GUARD_BEGIN
  set_error("");
  if (!h || !out) return fail(SAIGE_EINVAL, "null argument").code;
  if (n != h->n) return fail(SAIGE_EINVAL, "n mismatch").code;
  std::lock_guard<std::recursive_mutex> lk(h->mu);
  DeviceGuard dg(h->device);
  auto body = [&]() -> Status {
    SG_TRY(h->ws_io.reserve((size_t)h->n_pad * sizeof(double)));
    double* dd = h->ws_io.as<double>();
    SG_TRY(grm_diag(h, dd, h->stream));
    SG_TRY(download_block(h, dd, out, 1, h->stream));
    SG_CUDA(cudaStreamSynchronize(h->stream));
    return Status();
  };
  return body().code;
  SG_GUARD_END
}

static int32_t pcg_entry(saige_grm* h, const double* w, const double tau[2], const double* b,
                         const double* x0, double* x, int64_t n, int32_t nrhs,
                         const saige_pcg_options* opt, int32_t* iters, double* resid,
                         uint8_t* converged, bool w_inverse) {
  if (!h || !w || !tau || !b || !x) return fail(SAIGE_EINVAL, "null argument").code;
  if (n != h->n) return fail(SAIGE_EINVAL, "n mismatch (%lld vs %lld)", (long long)n,
                             (long long)h->n).code;
  if (nrhs <= 0) return fail(SAIGE_EINVAL, "nrhs must be positive").code;
  saige_pcg_options o = {1e-5, 500, SAIGE_PREC_FP32};
  if (opt) o = *opt;
  std::lock_guard<std::recursive_mutex> lk(h->mu);
  DeviceGuard dg(h->device);
  cudaStream_t st = h->stream;
  ReleaseScope rs(ReleaseMode::kStream, st);
  auto body = [&]() -> Status {
    const int64_t ld = h->n_pad;
    const size_t blk = (size_t)ld * nrhs;
    // io: b, x0, x (blocks) + wv, d (vectors)
    SG_TRY(h->ws_io.reserve((3 * blk + 3 * (size_t)ld) * sizeof(double)));
    double* db = h->ws_io.as<double>();
    double* dx0 = db + blk;
    double* dx = dx0 + blk;
    double* dw = dx + blk;
    double* dwv = dw + ld;
    double* dd = dwv + ld;
    SG_TRY(upload_block(h, b, db, nrhs, st));
    if (x0) SG_TRY(upload_block(h, x0, dx0, nrhs, st));
    SG_TRY(upload_block(h, w, dw, 1, st));
    if (w_inverse) {
      SG_CUDA(sigma_diag(dw, tau[0], tau[1], dwv, dd, h->n, st));
    } else {
      SG_CUDA(sigma_diag_w(dw, tau[0], tau[1], dd, h->n, st));
      SG_CUDA(cudaMemcpyAsync(dwv, dw, (size_t)ld * 8, cudaMemcpyDeviceToDevice, st));
    }
    PcgRun run;
    run.b = db;
    run.x0 = x0 ? dx0 : nullptr;
    run.wv = dwv;
    run.d = dd;
    run.tau0 = tau[0];
    run.tau1 = tau[1];
    run.w_inverse = w_inverse;
    run.q = nrhs;
    run.tol = o.tol;
    run.max_iter = o.max_iter;
    run.precision = o.precision;
    run.x = dx;
    SG_TRY(pcg_run(h, run, st));
    SG_TRY(download_block(h, dx, x, nrhs, st));
    SG_CUDA(cudaStreamSynchronize(st));
    for (int c = 0; c < nrhs; ++c) {
      if (iters) iters[c] = run.iters[(size_t)c];
      if (resid) resid[c] = run.resid[(size_t)c];
      if (converged) converged[c] = run.state[(size_t)c] == kColConverged ? 1 : 0;
    }
    return Status();
  };
  return body().code;
}

SG_API int32_t saige_pcg_solve(saige_grm* h, const double* w, const double tau[2], const double* b,
                               const double* x0, double* x, int64_t n, int32_t nrhs,
                               const saige_pcg_options* opt, int32_t* iters, double* resid,
                               uint8_t* converged) {
  SG_GUARD_BEGIN
  set_error("");
  return pcg_entry(h, w, tau, b, x0, x, n, nrhs, opt, iters, resid, converged, true);
  SG_GUARD_END
}

SG_API int32_t saige_solve_mixed_model_pcg(saige_grm* h, const double tau[2], const double* w,
                                           const double* b, double* x, int64_t n,
                                           const saige_pcg_options* opt, int32_t* iters,
                                           double* resid, uint8_t* converged) {
  SG_GUARD_BEGIN
  set_error("");
  return pcg_entry(h, w, tau, b, nullptr, x, n, 1, opt, iters, resid, converged, false);
  SG_GUARD_END
}
