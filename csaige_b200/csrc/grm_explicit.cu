// Explicit genetic relationship matrix: compute_dense_grm
// (saige-core/src/grm/dense.rs:22-112), compute_grm_from_dosages (dense.rs:115-186),
// compute_sparse_grm (grm/sparse.rs:18-66) and compute_sparse_grm_from_dosages
// (sparse.rs:69-98), with the .sparseGRM.mtx writer (saige-geno/src/
// sparse_grm_io.rs:73-115).
//
// K_ij = (1/M) sum_m z_im z_jm over the M used markers.  The reference forms each
// entry of the upper triangle as one f64 sum over the markers in file order,
// `val += gi * gj` (a rounded multiply, then a rounded add: rustc does not fuse
// them), and multiplies it by 1/M.  grm_syrk_kernel keeps exactly that order for
// every entry: a CTA owns a 128 x 128 tile of the upper triangle, each thread 8 x 8
// entries, and all of them walk the markers in file order with __dmul_rn and
// __dadd_rn, so the result is bit-identical to the reference's.  This is FP64 work
// on the CUDA cores: tcgen05 has no f64 kind, and a fixed-order sum of f64 products
// is not an integer problem the int8 tensor path could reproduce.  The FMA variant
// fuses each pair (twice the FP64 rate, last-bit differences).
//
// Operands come from the packed 2-bit rows (the device word layout of
// kernels_bed.cu) through a per-marker table of the four z values, so the genotype
// matrix is read at 2 bits per entry; the dosage entry point stages an f64 z matrix
// standardised on the device instead.  The sparse form thresholds in the epilogue
// (diagonal, or |K_ij| >= cutoff) and appends (i, j, K_ij) triplets with one atomic
// per warp, so the n x n matrix is never stored.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "engine.cuh"

struct saige_sparse_grm {
  int64_t n = 0;
  int64_t n_markers_used = 0;
  std::vector<int32_t> rows, cols;  // upper triangle with the diagonal, row-major
  std::vector<double> vals;
};

namespace saige {
namespace {

constexpr int kT = 128;    // samples per tile side
constexpr int kKc = 32;    // markers per shared-memory stage
constexpr int kThr = 256;  // 16 x 16 threads, 8 x 8 entries each
constexpr int kWordsSide = kT / 16;
constexpr size_t kSmemBytes = 2 * ((size_t)2 * kKc * kT * sizeof(double)   // z, both sides
                                   + (size_t)kKc * 4 * sizeof(double)       // z table
                                   + (size_t)2 * kKc * kWordsSide * 4);     // packed words

struct SyrkArgs {
  const uint32_t* geno = nullptr;  // packed rows (m_pad x wpr words), or
  int64_t wpr = 0;
  const double* lut = nullptr;     // 4 z values per marker, by 2-bit code
  const double* z = nullptr;       // f64 z rows (m_pad x ldz), zero padded
  int64_t ldz = 0;
  int64_t n = 0, m_pad = 0;        // samples; markers (a multiple of kKc, padding z = 0)
  const int2* tiles = nullptr;     // (bi, bj), bi <= bj
  double scale = 0.0;              // 1 / n_used (0 when no marker is used)
  double* dense = nullptr;         // n x n
  int32_t* rows = nullptr;         // sparse triplets
  int32_t* cols = nullptr;
  double* vals = nullptr;
  unsigned long long* count = nullptr;
  int64_t cap = 0;
  double cutoff = 0.0;
};

// Bit offset of entry e (0..15) of a packed word: e = 4j + i sits at
// 16*(j>>1) + 2*(j&1) + 4i (kernels_bed.cu, to_device_layout).
__device__ __forceinline__ int code_shift(int e) {
  const int j = e >> 2, i = e & 3;
  return 16 * (j >> 1) + 2 * (j & 1) + 4 * i;
}

template <bool kPacked, bool kFma, bool kSparse>
__global__ void __launch_bounds__(kThr, 1) grm_syrk_kernel(const SyrkArgs a) {
  // Two stages in flight: while the threads multiply stage c out of zs[c & 1], each
  // k-step also decodes 1/32 of stage c + 1 into zs[(c + 1) & 1], from the packed
  // words stored (before the previous barrier) in sraw[(c + 1) & 1]; the words of
  // stage c + 2 are loaded into registers at the start of stage c.  One barrier per
  // stage separates every write of a buffer from its reads.
  extern __shared__ __align__(16) double smem[];
  double* zs = smem;                       // [buf][side][k][s], side 0 = rows i, 1 = columns j
  double* slut = zs + 2 * 2 * kKc * kT;    // [buf][k][code]
  uint32_t* sraw = reinterpret_cast<uint32_t*>(slut + 2 * kKc * 4);  // [buf][side][k][word]
  constexpr int kZ = 2 * kKc * kT;         // doubles per z buffer
  constexpr int kRaw = 2 * kKc * kWordsSide;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int2 tile = a.tiles[blockIdx.x];
  const int64_t i0 = (int64_t)tile.x * kT, j0 = (int64_t)tile.y * kT;
  const int nch = (int)(a.m_pad / kKc);

  uint32_t wreg0 = 0, wreg1 = 0;
  double lreg = 0.0;
  // Packed source: thread t loads words v = t and v = t + 256 of stage q,
  // v = (side * kKc + k) * 8 + w, and table entry t of it (t < 128).
  auto fetch = [&](int q) {
    if constexpr (kPacked) {
      const int64_t row0 = (int64_t)q * kKc;
      {
        const int v = tid, side = v >> 8, k = (v >> 3) & (kKc - 1), w = v & 7;
        wreg0 = __ldg(a.geno + (row0 + k) * a.wpr + (side ? j0 : i0) / 16 + w);
      }
      {
        const int v = tid + kThr, side = v >> 8, k = (v >> 3) & (kKc - 1), w = v & 7;
        wreg1 = __ldg(a.geno + (row0 + k) * a.wpr + (side ? j0 : i0) / 16 + w);
      }
      if (tid < kKc * 4) lreg = __ldg(a.lut + row0 * 4 + tid);
    }
  };
  auto store_raw = [&](int q) {
    if constexpr (kPacked) {
      uint32_t* r = sraw + (q & 1) * kRaw;
      r[tid] = wreg0;
      r[tid + kThr] = wreg1;
      if (tid < kKc * 4) slut[(q & 1) * kKc * 4 + tid] = lreg;
    }
  };
  // Decode slice `it` (0..31) of stage q: entry v = tid + 256 it of its z buffer,
  // v = (side * kKc + k) * kT + s.
  auto decode = [&](int q, int it) {
    const int v = tid + it * kThr;
    const int k = (v >> 7) & (kKc - 1), s = v & (kT - 1);
    double* z = zs + (q & 1) * kZ;
    if constexpr (kPacked) {
      const uint32_t word = sraw[(q & 1) * kRaw + (v >> 7) * kWordsSide + (s >> 4)];
      z[v] = slut[(q & 1) * kKc * 4 + k * 4 + ((word >> code_shift(s & 15)) & 3u)];
    } else {
      const int side = v >> 12;
      z[v] = __ldg(a.z + ((int64_t)q * kKc + k) * a.ldz + (side ? j0 : i0) + s);
    }
  };

  double acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[r][q] = 0.0;

  // prologue: stage 0 decoded, the words of stage 1 in shared memory
  fetch(0);
  store_raw(0);
  if (nch > 1) fetch(1);
  __syncthreads();
#pragma unroll 4
  for (int it = 0; it < kKc; ++it) decode(0, it);
  if (nch > 1) store_raw(1);
  __syncthreads();

  for (int c = 0; c < nch; ++c) {
    const bool next = c + 1 < nch;
    if (c + 2 < nch) fetch(c + 2);
    const double* zi = zs + (c & 1) * kZ + ty;
    const double* zj = zs + (c & 1) * kZ + kKc * kT + tx;
#pragma unroll 2
    for (int k = 0; k < kKc; ++k) {
      double x[8], y[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) x[r] = zi[k * kT + 16 * r];
#pragma unroll
      for (int q = 0; q < 8; ++q) y[q] = zj[k * kT + 16 * q];
      if (next) decode(c + 1, k);
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          if constexpr (kFma)
            acc[r][q] = __fma_rn(x[r], y[q], acc[r][q]);
          else
            acc[r][q] = __dadd_rn(acc[r][q], __dmul_rn(x[r], y[q]));
        }
    }
    // sraw[c & 1] was last read while stage c was decoded, before the previous barrier
    if (c + 2 < nch) store_raw(c + 2);
    __syncthreads();
  }

  const bool diag = tile.x == tile.y;
  const int lane = tid & 31;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int64_t gi = i0 + ty + 16 * r;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int64_t gj = j0 + tx + 16 * q;
      const double v = acc[r][q] * a.scale;  // dense.rs:91-95, val * scale
      if constexpr (!kSparse) {
        if (gi < a.n && gj < a.n) {
          a.dense[gi * a.n + gj] = v;
          if (!diag) a.dense[gj * a.n + gi] = v;
        }
      } else {
        // sparse.rs:40-44: the diagonal, or |K_ij| >= cutoff, of the upper triangle
        const bool keep = gi < a.n && gj < a.n && gi <= gj && (gi == gj || fabs(v) >= a.cutoff);
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (mask) {
          const int leader = __ffs(mask) - 1;
          unsigned long long base = 0;
          if (lane == leader) base = atomicAdd(a.count, (unsigned long long)__popc(mask));
          base = __shfl_sync(0xffffffffu, base, leader);
          if (keep) {
            const unsigned long long slot = base + __popc(mask & ((1u << lane) - 1u));
            if (slot < (unsigned long long)a.cap) {
              a.rows[slot] = (int32_t)gi;
              a.cols[slot] = (int32_t)gj;
              a.vals[slot] = v;
            }
          }
        }
      }
    }
  }
}

// z[k][i] = (d - mean_k) / sd_k with a missing call at the mean (dense.rs:129-140),
// for the used rows; zero for padding rows and samples.
__global__ void grm_standardize_kernel(const double* __restrict__ dos, int64_t n,
                                       const int64_t* __restrict__ rows,
                                       const double* __restrict__ mean,
                                       const double* __restrict__ sd, int64_t m_used,
                                       int64_t m_pad, int64_t n_pad, double* __restrict__ z) {
  for (int64_t k = blockIdx.y; k < m_pad; k += gridDim.y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pad;
         i += (int64_t)gridDim.x * blockDim.x) {
      double out = 0.0;
      if (k < m_used && i < n) {
        double d = dos[rows[k] * n + i];
        const double mu = mean[k];
        if (isnan(d)) d = mu;
        out = __ddiv_rn(__dsub_rn(d, mu), sd[k]);
      }
      z[k * n_pad + i] = out;
    }
  }
}

template <bool kPacked, bool kFma, bool kSparse>
cudaError_t launch_syrk_t(const SyrkArgs& a, int64_t n_tiles, cudaStream_t st) {
  auto k = grm_syrk_kernel<kPacked, kFma, kSparse>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmemBytes);
  if (e != cudaSuccess) return e;
  k<<<(unsigned)n_tiles, kThr, kSmemBytes, st>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_syrk(const SyrkArgs& a, bool packed, bool fma, bool sparse, int64_t n_tiles,
                        cudaStream_t st) {
  if (packed) {
    if (fma) return sparse ? launch_syrk_t<true, true, true>(a, n_tiles, st)
                           : launch_syrk_t<true, true, false>(a, n_tiles, st);
    return sparse ? launch_syrk_t<true, false, true>(a, n_tiles, st)
                  : launch_syrk_t<true, false, false>(a, n_tiles, st);
  }
  if (fma) return sparse ? launch_syrk_t<false, true, true>(a, n_tiles, st)
                         : launch_syrk_t<false, true, false>(a, n_tiles, st);
  return sparse ? launch_syrk_t<false, false, true>(a, n_tiles, st)
                : launch_syrk_t<false, false, false>(a, n_tiles, st);
}

struct Stream {
  cudaStream_t s = nullptr;
  ~Stream() {
    if (s) cudaStreamDestroy(s);
  }
};

struct Events {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~Events() {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

// Runs the SYRK over a prepared source and collects the dense matrix (host, n x n)
// or the sparse triplets (sorted row-major).  a: source fields set.
Status run_syrk(SyrkArgs a, int64_t n, int64_t n_pad, bool packed, int32_t arith, double cutoff,
                double* dense_host, saige_sparse_grm* sp, cudaStream_t st, double* kernel_s) {
  const int64_t nb = n_pad / kT;
  std::vector<int2> tiles;
  tiles.reserve((size_t)(nb * (nb + 1) / 2));
  for (int64_t bi = 0; bi < nb; ++bi)
    for (int64_t bj = bi; bj < nb; ++bj) tiles.push_back(make_int2((int)bi, (int)bj));
  const int64_t n_tiles = (int64_t)tiles.size();
  if (n_tiles > INT32_MAX) return fail(SAIGE_EINVAL, "too many sample tiles");
  DevBuf d_tiles;
  SG_TRY(d_tiles.reserve(tiles.size() * sizeof(int2)));
  SG_CUDA(cudaMemcpyAsync(d_tiles.ptr, tiles.data(), tiles.size() * sizeof(int2),
                          cudaMemcpyHostToDevice, st));
  a.tiles = d_tiles.as<int2>();
  a.n = n;
  a.cutoff = cutoff;
  const bool fma = arith == SAIGE_GRM_ARITH_FMA;
  Events ev;
  SG_CUDA(cudaEventCreate(&ev.e0));
  SG_CUDA(cudaEventCreate(&ev.e1));
  double ktime = 0.0;
  auto timed_launch = [&](bool sparse) -> Status {
    SG_CUDA(cudaEventRecord(ev.e0, st));
    SG_CUDA(launch_syrk(a, packed, fma, sparse, n_tiles, st));
    SG_CUDA(cudaEventRecord(ev.e1, st));
    SG_CUDA(cudaEventSynchronize(ev.e1));
    float ms = 0.f;
    SG_CUDA(cudaEventElapsedTime(&ms, ev.e0, ev.e1));
    ktime += ms * 1e-3;
    return Status();
  };
  if (!sp) {
    DevBuf d_out;
    SG_TRY(d_out.reserve((size_t)n * n * sizeof(double)));
    a.dense = d_out.as<double>();
    SG_TRY(timed_launch(false));
    SG_CUDA(cudaMemcpyAsync(dense_host, d_out.ptr, (size_t)n * n * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
  } else {
    DevBuf d_cnt, d_rows, d_cols, d_vals;
    SG_TRY(d_cnt.reserve(sizeof(unsigned long long)));
    int64_t cap = n * 16 + 4096;
    unsigned long long cnt = 0;
    for (int attempt = 0; attempt < 2; ++attempt) {
      SG_TRY(d_rows.reserve((size_t)cap * sizeof(int32_t)));
      SG_TRY(d_cols.reserve((size_t)cap * sizeof(int32_t)));
      SG_TRY(d_vals.reserve((size_t)cap * sizeof(double)));
      SG_CUDA(cudaMemsetAsync(d_cnt.ptr, 0, sizeof(unsigned long long), st));
      a.rows = d_rows.as<int32_t>();
      a.cols = d_cols.as<int32_t>();
      a.vals = d_vals.as<double>();
      a.count = d_cnt.as<unsigned long long>();
      a.cap = cap;
      SG_TRY(timed_launch(true));
      SG_CUDA(cudaMemcpyAsync(&cnt, d_cnt.ptr, sizeof(cnt), cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaStreamSynchronize(st));
      if ((int64_t)cnt <= cap) break;
      // more entries passed the cutoff than the first guess holds: size exactly and redo
      cap = (int64_t)cnt;
      d_rows.release();
      d_cols.release();
      d_vals.release();
    }
    if ((int64_t)cnt > cap) return fail(SAIGE_EINVAL, "sparse GRM size changed between passes");
    const size_t nnz = (size_t)cnt;
    std::vector<int32_t> r(nnz), c(nnz);
    std::vector<double> v(nnz);
    if (nnz) {
      SG_CUDA(cudaMemcpyAsync(r.data(), d_rows.ptr, nnz * 4, cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaMemcpyAsync(c.data(), d_cols.ptr, nnz * 4, cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaMemcpyAsync(v.data(), d_vals.ptr, nnz * 8, cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaStreamSynchronize(st));
    }
    // the writer's order (sparse_grm_io.rs:92-107): by row, then column
    std::vector<uint64_t> key(nnz);
    for (size_t e = 0; e < nnz; ++e) key[e] = ((uint64_t)(uint32_t)r[e] << 32) | (uint32_t)c[e];
    std::vector<size_t> perm(nnz);
    for (size_t e = 0; e < nnz; ++e) perm[e] = e;
    std::sort(perm.begin(), perm.end(), [&](size_t x, size_t y) { return key[x] < key[y]; });
    sp->rows.resize(nnz);
    sp->cols.resize(nnz);
    sp->vals.resize(nnz);
    for (size_t e = 0; e < nnz; ++e) {
      sp->rows[e] = r[perm[e]];
      sp->cols[e] = c[perm[e]];
      sp->vals[e] = v[perm[e]];
    }
    sp->n = n;
  }
  if (kernel_s) *kernel_s = ktime;
  return Status();
}

Status check_config(const saige_explicit_grm_config* cfg) {
  if (!cfg) return fail(SAIGE_EINVAL, "null config");
  if (cfg->arith != SAIGE_GRM_ARITH_REFERENCE && cfg->arith != SAIGE_GRM_ARITH_FMA)
    return fail(SAIGE_EINVAL, "unknown arith %d", cfg->arith);
  if (std::isnan(cfg->min_maf) || std::isnan(cfg->relatedness_cutoff))
    return fail(SAIGE_EINVAL, "min_maf and relatedness_cutoff must not be NaN");
  return Status();
}

void fill_info(saige_explicit_grm_info* info, int64_t n, int64_t used, int64_t nnz, double ks,
               double total_s) {
  if (!info) return;
  info->n_markers_used = used;
  info->nnz = nnz;
  info->kernel_seconds = ks;
  info->total_seconds = total_s;
  info->terms = (double)n * (double)(n + 1) / 2.0 * (double)used;
}

// compute_dense_grm / compute_sparse_grm on a host .bed.
Status grm_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                    const int64_t* sample_idx, int64_t n, const saige_explicit_grm_config* cfg,
                    double* dense_out, saige_sparse_grm* sp, saige_explicit_grm_info* info) {
  const auto t0 = std::chrono::steady_clock::now();
  SG_TRY(check_config(cfg));
  if (!bed) return fail(SAIGE_EINVAL, "null bed");
  if (m_tot < 0) return fail(SAIGE_EINVAL, "m_tot must be non-negative");
  int dev = 0;
  SG_TRY(pick_device(cfg->device, &dev));
  SG_TRY(check_bed_header(bed, bed_len, n_fam, m_tot));
  std::vector<int32_t> sidx;
  bool identity = true;
  SG_TRY(check_subset(sample_idx, n, n_fam, sidx, identity));
  if (n > INT32_MAX) return fail(SAIGE_EINVAL, "n exceeds 2^31-1");
  const int64_t bpm = (n_fam + 3) / 4;
  const size_t used_bytes = (size_t)(3 + bpm * m_tot);
  Stream stream;
  SG_CUDA(cudaStreamCreateWithFlags(&stream.s, cudaStreamNonBlocking));
  cudaStream_t st = stream.s;

  DevBuf d_bed, d_cnt;
  SG_TRY(d_bed.reserve(used_bytes));
  SG_CUDA(cudaMemcpyAsync(d_bed.ptr, bed, used_bytes, cudaMemcpyHostToDevice, st));
  // af of every marker (traits.rs:42-54 from exact integer counts)
  std::vector<int64_t> all((size_t)m_tot);
  for (int64_t j = 0; j < m_tot; ++j) all[(size_t)j] = j;
  std::vector<int64_t> cnt((size_t)m_tot * 2);
  if (m_tot > 0) {
    SG_TRY(d_cnt.reserve((size_t)m_tot * 2 * sizeof(int64_t)));
    SG_TRY(bed_gather_dev(d_bed.as<uint8_t>(), n_fam, all, sidx, identity, n, nullptr, 0,
                          d_cnt.as<int64_t>(), st));
    SG_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt.ptr, cnt.size() * 8, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    d_cnt.release();
  }
  // dense.rs:34-58: the af window, the variance floor, and the z of each code
  // (00 -> 2, 01 -> missing at the mean, 10 -> 1, 11 -> 0)
  std::vector<int64_t> used;
  std::vector<double> lut;
  for (int64_t j = 0; j < m_tot; ++j) {
    const int64_t alt = cnt[(size_t)(2 * j)], nv = n - cnt[(size_t)(2 * j + 1)];
    const double af = nv > 0 ? (double)alt / (2.0 * (double)nv) : 0.0;
    if (af < cfg->min_maf || af > 1.0 - cfg->min_maf) continue;
    const double var = 2.0 * af * (1.0 - af);
    if (var < 1e-10) continue;
    const double sd = std::sqrt(var);
    const double mean = 2.0 * af;
    used.push_back(j);
    lut.push_back((2.0 - mean) / sd);
    lut.push_back((mean - mean) / sd);
    lut.push_back((1.0 - mean) / sd);
    lut.push_back((0.0 - mean) / sd);
  }
  const int64_t m_used = (int64_t)used.size();
  const int64_t m_pad = std::max<int64_t>(round_up(m_used, kKc), kKc);
  lut.resize((size_t)m_pad * 4, 0.0);
  const int64_t n_pad = round_up(n, kT), wpr = n_pad / 16;
  DevBuf d_geno, d_lut;
  SG_TRY(d_geno.reserve((size_t)m_pad * wpr * 4));
  SG_CUDA(cudaMemsetAsync(d_geno.ptr, 0, (size_t)m_pad * wpr * 4, st));
  if (m_used > 0)
    SG_TRY(bed_gather_dev(d_bed.as<uint8_t>(), n_fam, used, sidx, identity, n,
                          d_geno.as<uint32_t>(), wpr, nullptr, st));
  d_bed.release();
  SG_TRY(d_lut.reserve(lut.size() * sizeof(double)));
  SG_CUDA(cudaMemcpyAsync(d_lut.ptr, lut.data(), lut.size() * sizeof(double),
                          cudaMemcpyHostToDevice, st));
  SyrkArgs a;
  a.geno = d_geno.as<uint32_t>();
  a.wpr = wpr;
  a.lut = d_lut.as<double>();
  a.m_pad = m_pad;
  a.scale = m_used > 0 ? 1.0 / (double)m_used : 0.0;
  double ks = 0.0;
  SG_TRY(run_syrk(a, n, n_pad, true, cfg->arith, cfg->relatedness_cutoff, dense_out, sp, st, &ks));
  if (sp) sp->n_markers_used = m_used;
  const double tot =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  fill_info(info, n, m_used, sp ? (int64_t)sp->vals.size() : n * n, ks, tot);
  return Status();
}

// compute_grm_from_dosages / compute_sparse_grm_from_dosages.
Status grm_from_dosages(const double* dos, const double* af, int64_t n, int64_t m,
                        const saige_explicit_grm_config* cfg, double* dense_out,
                        saige_sparse_grm* sp, saige_explicit_grm_info* info) {
  const auto t0 = std::chrono::steady_clock::now();
  SG_TRY(check_config(cfg));
  if (m < 0 || n < 0 || (m > 0 && (!dos || !af)))
    return fail(SAIGE_EINVAL, "null argument or negative size");
  if (m == 0 || n == 0) {
    // dense.rs:117-120: no marker rows give the 0 x 0 matrix
    if (sp) sp->n = 0;
    fill_info(info, 0, 0, 0, 0.0, 0.0);
    return Status();
  }
  if (n > INT32_MAX) return fail(SAIGE_EINVAL, "n exceeds 2^31-1");
  int dev = 0;
  SG_TRY(pick_device(cfg->device, &dev));
  std::vector<int64_t> used;
  std::vector<double> mean, sd;
  for (int64_t j = 0; j < m; ++j) {
    const double var = 2.0 * af[j] * (1.0 - af[j]);  // dense.rs:125-130
    if (var < 1e-10) continue;
    used.push_back(j);
    sd.push_back(std::sqrt(var));
    mean.push_back(2.0 * af[j]);
  }
  const int64_t m_used = (int64_t)used.size();
  const int64_t m_pad = std::max<int64_t>(round_up(m_used, kKc), kKc);
  const int64_t n_pad = round_up(n, kT);
  Stream stream;
  SG_CUDA(cudaStreamCreateWithFlags(&stream.s, cudaStreamNonBlocking));
  cudaStream_t st = stream.s;
  DevBuf d_dos, d_rows, d_mean, d_sd, d_z;
  SG_TRY(d_z.reserve((size_t)m_pad * n_pad * sizeof(double)));
  if (m_used > 0) {
    SG_TRY(d_dos.reserve((size_t)m * n * sizeof(double)));
    SG_TRY(d_rows.reserve((size_t)m_used * sizeof(int64_t)));
    SG_TRY(d_mean.reserve((size_t)m_used * sizeof(double)));
    SG_TRY(d_sd.reserve((size_t)m_used * sizeof(double)));
    SG_CUDA(cudaMemcpyAsync(d_dos.ptr, dos, (size_t)m * n * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(d_rows.ptr, used.data(), (size_t)m_used * 8, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(d_mean.ptr, mean.data(), (size_t)m_used * 8, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(d_sd.ptr, sd.data(), (size_t)m_used * 8, cudaMemcpyHostToDevice, st));
  }
  const dim3 grid((unsigned)std::min<int64_t>(ceil_div(n_pad, 256), 1024),
                  (unsigned)std::min<int64_t>(m_pad, 65535));
  grm_standardize_kernel<<<grid, 256, 0, st>>>(d_dos.as<double>(), n, d_rows.as<int64_t>(),
                                               d_mean.as<double>(), d_sd.as<double>(), m_used,
                                               m_pad, n_pad, d_z.as<double>());
  count_launches(1);
  SG_CHECK_LAUNCH();
  SyrkArgs a;
  a.z = d_z.as<double>();
  a.ldz = n_pad;
  a.m_pad = m_pad;
  a.scale = m_used > 0 ? 1.0 / (double)m_used : 0.0;
  double ks = 0.0;
  SG_TRY(run_syrk(a, n, n_pad, false, cfg->arith, cfg->relatedness_cutoff, dense_out, sp, st,
                  &ks));
  if (sp) sp->n_markers_used = m_used;
  const double tot =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  fill_info(info, n, m_used, sp ? (int64_t)sp->vals.size() : n * n, ks, tot);
  return Status();
}

}  // namespace
}  // namespace saige

using namespace saige;

#define SG_API extern "C" __attribute__((visibility("default")))

#define SG_GUARD_BEGIN try {
#define SG_GUARD_END                                          \
  }                                                           \
  catch (const std::bad_alloc&) {                             \
    return fail(SAIGE_ENOMEM, "host allocation failed").code; \
  }                                                           \
  catch (...) {                                               \
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code; \
  }

SG_API int32_t saige_explicit_grm_config_default(saige_explicit_grm_config* cfg) {
  if (!cfg) return fail(SAIGE_EINVAL, "null config").code;
  memset(cfg, 0, sizeof(*cfg));
  cfg->min_maf = 0.01;             // create_sparse_grm.rs:28-30
  cfg->relatedness_cutoff = 0.125;  // create_sparse_grm.rs:24-26
  cfg->arith = SAIGE_GRM_ARITH_REFERENCE;
  cfg->device = -1;
  return SAIGE_OK;
}

SG_API int32_t saige_dense_grm_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                        int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                        const saige_explicit_grm_config* cfg, double* out,
                                        saige_explicit_grm_info* info) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out) return fail(SAIGE_EINVAL, "null output").code;
  return grm_from_bed(bed, bed_len, n_fam, m_tot, sample_idx, n, cfg, out, nullptr, info).code;
  SG_GUARD_END
}

SG_API int32_t saige_sparse_grm_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                         int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                         const saige_explicit_grm_config* cfg,
                                         saige_sparse_grm** out, saige_explicit_grm_info* info) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out) return fail(SAIGE_EINVAL, "null output").code;
  *out = nullptr;
  auto* g = new saige_sparse_grm();
  const Status s = grm_from_bed(bed, bed_len, n_fam, m_tot, sample_idx, n, cfg, nullptr, g, info);
  if (!s.ok()) {
    delete g;
    return s.code;
  }
  *out = g;
  return SAIGE_OK;
  SG_GUARD_END
}

SG_API int32_t saige_grm_from_dosages(const double* dosages, const double* af, int64_t n,
                                      int64_t m, const saige_explicit_grm_config* cfg,
                                      double* out, saige_explicit_grm_info* info) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out && m > 0 && n > 0) return fail(SAIGE_EINVAL, "null output").code;
  return grm_from_dosages(dosages, af, n, m, cfg, out, nullptr, info).code;
  SG_GUARD_END
}

SG_API int32_t saige_sparse_grm_from_dosages(const double* dosages, const double* af, int64_t n,
                                             int64_t m, const saige_explicit_grm_config* cfg,
                                             saige_sparse_grm** out,
                                             saige_explicit_grm_info* info) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out) return fail(SAIGE_EINVAL, "null output").code;
  *out = nullptr;
  auto* g = new saige_sparse_grm();
  const Status s = grm_from_dosages(dosages, af, n, m, cfg, nullptr, g, info);
  if (!s.ok()) {
    delete g;
    return s.code;
  }
  *out = g;
  return SAIGE_OK;
  SG_GUARD_END
}

SG_API int64_t saige_sparse_grm_n(const saige_sparse_grm* g) { return g ? g->n : -1; }

SG_API int64_t saige_sparse_grm_nnz(const saige_sparse_grm* g) {
  return g ? (int64_t)g->vals.size() : -1;
}

SG_API int64_t saige_sparse_grm_n_markers(const saige_sparse_grm* g) {
  return g ? g->n_markers_used : -1;
}

SG_API int32_t saige_sparse_grm_get(const saige_sparse_grm* g, int32_t* rows, int32_t* cols,
                                    double* vals) {
  SG_GUARD_BEGIN
  if (!g) return fail(SAIGE_EINVAL, "null handle").code;
  const size_t nnz = g->vals.size();
  if (nnz && (!rows || !cols || !vals)) return fail(SAIGE_EINVAL, "null output").code;
  if (nnz) {
    memcpy(rows, g->rows.data(), nnz * 4);
    memcpy(cols, g->cols.data(), nnz * 4);
    memcpy(vals, g->vals.data(), nnz * 8);
  }
  return SAIGE_OK;
  SG_GUARD_END
}

SG_API void saige_sparse_grm_free(saige_sparse_grm* g) { delete g; }

SG_API int32_t saige_sparse_grm_from_triplets(int64_t n, int64_t nnz, const int32_t* rows,
                                              const int32_t* cols, const double* vals,
                                              int64_t n_markers_used, saige_sparse_grm** out) {
  SG_GUARD_BEGIN
  set_error("");
  if (!out || n < 0 || nnz < 0 || (nnz > 0 && (!rows || !cols || !vals)))
    return fail(SAIGE_EINVAL, "null argument or negative size").code;
  *out = nullptr;
  for (int64_t e = 0; e < nnz; ++e) {
    if (rows[e] < 0 || rows[e] > cols[e] || cols[e] >= n)
      return fail(SAIGE_EINVAL, "entry %lld (%d, %d) is not in the upper triangle of %lld x %lld",
                  (long long)e, rows[e], cols[e], (long long)n, (long long)n).code;
    if (e > 0 && (rows[e] < rows[e - 1] || (rows[e] == rows[e - 1] && cols[e] <= cols[e - 1])))
      return fail(SAIGE_EINVAL, "entries must be sorted by row, then column, without repeats").code;
  }
  auto* g = new saige_sparse_grm();
  g->n = n;
  g->n_markers_used = n_markers_used;
  g->rows.assign(rows, rows + nnz);
  g->cols.assign(cols, cols + nnz);
  g->vals.assign(vals, vals + nnz);
  *out = g;
  return SAIGE_OK;
  SG_GUARD_END
}

SG_API int32_t saige_write_sparse_grm(const saige_sparse_grm* g, const char* const* sample_ids,
                                      int64_t n_ids, const char* mtx_path, const char* ids_path) {
  SG_GUARD_BEGIN
  set_error("");
  if (!g || !mtx_path || !ids_path || n_ids < 0 || (n_ids > 0 && !sample_ids))
    return fail(SAIGE_EINVAL, "null argument").code;
  // sample IDs, one per line (sparse_grm_io.rs:81-85)
  FILE* f = fopen(ids_path, "wb");
  if (!f) return fail(SAIGE_EINVAL, "cannot open %s for writing", ids_path).code;
  bool ok = true;
  for (int64_t i = 0; i < n_ids && ok; ++i) ok = fprintf(f, "%s\n", sample_ids[i]) >= 0;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(SAIGE_EINVAL, "writing %s failed", ids_path).code;
  // header, "n n nnz", then 1-based "i j value" with 10 decimals (:88-112)
  f = fopen(mtx_path, "wb");
  if (!f) return fail(SAIGE_EINVAL, "cannot open %s for writing", mtx_path).code;
  ok = fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n%lld %lld %lld\n",
               (long long)g->n, (long long)g->n, (long long)g->vals.size()) >= 0;
  for (size_t e = 0; e < g->vals.size() && ok; ++e)
    ok = fprintf(f, "%d %d %.10f\n", g->rows[e] + 1, g->cols[e] + 1, g->vals[e]) >= 0;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return fail(SAIGE_EINVAL, "writing %s failed", mtx_path).code;
  return SAIGE_OK;
  SG_GUARD_END
}
