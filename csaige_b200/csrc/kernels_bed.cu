// K1: gather the sample subset out of raw PLINK .bed rows, repack it into
// 128-byte-aligned 2-bit rows (device word layout, see to_device_layout), and
// count alleles and missing calls exactly.
//
// Replaces PlinkReader::read_marker_raw / read_marker (saige-geno/src/
// plink.rs:182-194, 237-249) and MarkerData::compute_af's sums
// (saige-geno/src/traits.rs:42-54): the counts are integers from popc over
// the code bit planes, so af = alt / (2 n_valid) computed from them on the
// host is bit-identical to the reference's f64 sum of 0/1/2 dosages.
#include "common.cuh"
#include "kernels.cuh"

namespace saige {

namespace {

constexpr int kThreads = 256;
constexpr int64_t kSmemRowMax = 200 * 1024;  // stage raw rows up to this size in shared memory

// Counts over a word of 16 codes; valid = even bits of the real samples.
__device__ __forceinline__ void count_word(uint32_t w, uint32_t valid, long long& alt,
                                           long long& miss) {
  const uint32_t lo = w & 0x55555555u;
  const uint32_t hi = (w >> 1) & 0x55555555u;
  const uint32_t hom_a1 = ~lo & ~hi & valid;  // 00 -> 2 copies of A1
  const uint32_t het = ~lo & hi & valid;      // 10 -> 1 copy
  const uint32_t mis = lo & ~hi & valid;      // 01 -> missing
  alt += 2 * __popc(hom_a1) + __popc(het);
  miss += __popc(mis);
}

// Device layout of a 32-bit word of 16 codes.  PLINK puts sample s at bits
// 2s; the packed rows put sample s = 4j + i at bit 16*(j>>1) + 2*(j&1) + 4i, so
// that each 4-sample group's codes sit in the low bits of four nibbles that one
// mask (or shift + mask) turns into a byte-permute selector.
__device__ __forceinline__ uint32_t nibble_spread16x2(uint32_t x) {
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  return (x | (x << 2)) & 0x33333333u;
}
__device__ __forceinline__ uint32_t to_device_layout(uint32_t plink_word) {
  return nibble_spread16x2(plink_word & 0x00FF00FFu) |
         (nibble_spread16x2((plink_word >> 8) & 0x00FF00FFu) << 2);
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Stages raw row `row` (bpm bytes) in shared memory in 16-byte chunks of its aligned
// span (row byte b at row_s[off + b]); the chunks that reach past either end of the
// row, at most two, are copied byte by byte, so no load leaves the row.  Several
// independent chunk loads per thread are in flight at once.  Returns row_s + off.
// row_s holds round_up(bpm + 16, 16) bytes, 16-byte aligned.
__device__ __forceinline__ const uint8_t* stage_row(const uint8_t* row, int64_t bpm,
                                                    uint8_t* row_s) {
  const int off = (int)(reinterpret_cast<uintptr_t>(row) & 15u);
  const uint4* base = reinterpret_cast<const uint4*>(row - off);
  const int64_t n16 = (off + bpm + 15) / 16;
#pragma unroll 4
  for (int64_t i = threadIdx.x; i < n16; i += blockDim.x) {
    const int64_t lo = 16 * i - off;
    if (lo >= 0 && lo + 16 <= bpm) {
      reinterpret_cast<uint4*>(row_s)[i] = __ldg(base + i);
    } else {
      for (int k = 0; k < 16; ++k) {
        const int64_t b = lo + k;
        if (b >= 0 && b < bpm) row_s[16 * i + k] = row[b];
      }
    }
  }
  __syncthreads();
  return row_s + off;
}

// The codes of samples sidx[0 .. kn) (kn <= 16) of a raw row as one PLINK-order
// word (sample k at bits 2k); vec: sidx is 16-byte aligned and kn == 16, so the
// indices are read as four 16-byte loads.
__device__ __forceinline__ uint32_t gather_word(const uint8_t* src, const int32_t* sidx, int kn,
                                                bool vec) {
  uint32_t word = 0;
  if (vec) {
    const int4* s4 = reinterpret_cast<const int4*>(sidx);
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int4 v = __ldg(s4 + g);
      const int32_t ss[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const uint32_t code = (src[ss[e] >> 2] >> ((ss[e] & 3) * 2)) & 3u;
        word |= code << (2 * (4 * g + e));
      }
    }
  } else {
    for (int k = 0; k < kn; ++k) {
      const int32_t s = sidx[k];
      const uint32_t code = (src[s >> 2] >> ((s & 3) * 2)) & 3u;
      word |= code << (2 * k);
    }
  }
  return word;
}

template <bool kIdentity>
__global__ void __launch_bounds__(kThreads)
    bed_gather_kernel(const uint8_t* __restrict__ bed, int64_t bpm,
                      const int64_t* __restrict__ src_rows, const int32_t* __restrict__ sidx,
                      int64_t n, uint32_t* __restrict__ out, int64_t wpr,
                      int64_t* __restrict__ counts, int use_smem) {
  extern __shared__ __align__(16) uint8_t row_s[];
  __shared__ long long red[2][kThreads / 32];
  const int64_t r = blockIdx.x;
  const uint8_t* row = bed + 3 + src_rows[r] * bpm;
  const uint8_t* src = use_smem ? stage_row(row, bpm, row_s) : row;
  const bool sidx16 = (reinterpret_cast<uintptr_t>(sidx) & 15u) == 0;
  long long alt = 0, miss = 0;
  const int64_t n_words_real = (n + 15) / 16;
  const int64_t n_words = out ? wpr : n_words_real;
  for (int64_t j = threadIdx.x; j < n_words; j += blockDim.x) {
    // Padding samples are coded 11 (genotype 0, not missing): every vector the
    // products read is zero there, so they contribute nothing to any sum.
    uint32_t w = 0xFFFFFFFFu;
    if (j < n_words_real) {
      const int64_t k0 = j * 16;
      const int kn = (n - k0) < 16 ? (int)(n - k0) : 16;
      uint32_t word = 0;
      if (kIdentity) {
        // bytes 4j .. 4j+3 of the raw row hold exactly these samples
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int64_t bi = 4 * j + b;
          const uint32_t byte = bi < bpm ? (uint32_t)src[bi] : 0u;
          word |= byte << (8 * b);
        }
      } else {
        word = gather_word(src, sidx + k0, kn, kn == 16 && sidx16);
      }
      const uint32_t keep = kn >= 16 ? 0xFFFFFFFFu : ((1u << (2 * kn)) - 1u);
      count_word(word, keep & 0x55555555u, alt, miss);
      // padding samples are coded 11, then the word is re-laid out
      w = to_device_layout((word & keep) | ~keep);
    }
    if (out) out[r * wpr + j] = w;
  }
  if (!counts) return;
  alt = warp_sum_ll(alt);
  miss = warp_sum_ll(miss);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][wid] = alt;
    red[1][wid] = miss;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long a = 0, mm = 0;
    for (int k = 0; k < kThreads / 32; ++k) {
      a += red[0][k];
      mm += red[1][k];
    }
    counts[2 * r] = a;
    counts[2 * r + 1] = mm;
  }
}

// Counts of several sample subsets ("cohorts") of the same raw rows in one pass:
// block = marker j0 + blockIdx.x, staged once in shared memory; for cohort c, the
// samples sidx[offs[c] .. offs[c] + n_c) (offs[c] a multiple of 16) are gathered 16 at
// a time and counted as bed_gather_kernel counts them.  counts[(c m_tot + j) 2 + e]:
// e = 0 alt-allele count, 1 missing count.
__global__ void __launch_bounds__(kThreads)
    bed_count_cohorts_kernel(const uint8_t* __restrict__ bed, int64_t bpm, int64_t j0,
                             const int32_t* __restrict__ sidx, const int64_t* __restrict__ offs,
                             const int64_t* __restrict__ ns, int n_cohorts, int64_t m_tot,
                             long long* __restrict__ counts) {
  extern __shared__ __align__(16) uint8_t row_s[];
  __shared__ long long red[2][kThreads / 32];
  const int64_t j = j0 + blockIdx.x;
  const uint8_t* src = stage_row(bed + 3 + j * bpm, bpm, row_s);
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = 0; c < n_cohorts; ++c) {
    const int32_t* sc = sidx + offs[c];
    const int64_t n = ns[c];
    const bool vec = (reinterpret_cast<uintptr_t>(sc) & 15u) == 0;
    long long alt = 0, miss = 0;
    for (int64_t w = threadIdx.x; w < (n + 15) / 16; w += blockDim.x) {
      const int64_t k0 = 16 * w;
      const int kn = (n - k0) < 16 ? (int)(n - k0) : 16;
      const uint32_t word = gather_word(src, sc + k0, kn, vec && kn == 16);
      const uint32_t keep = kn >= 16 ? 0xFFFFFFFFu : ((1u << (2 * kn)) - 1u);
      count_word(word, keep & 0x55555555u, alt, miss);
    }
    alt = warp_sum_ll(alt);
    miss = warp_sum_ll(miss);
    if (lane == 0) {
      red[0][wid] = alt;
      red[1][wid] = miss;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      long long a = 0, mm = 0;
      for (int k = 0; k < kThreads / 32; ++k) {
        a += red[0][k];
        mm += red[1][k];
      }
      counts[2 * ((int64_t)c * m_tot + j)] = a;
      counts[2 * ((int64_t)c * m_tot + j) + 1] = mm;
    }
    __syncthreads();  // red is reused by the next cohort
  }
}

// The packed rows of several sample subsets from one pass over the raw rows: block =
// rpb consecutive raw markers from j0 + blockIdx.x rpb, staged once; for every cohort,
// each thread loads the sample indices of a 16-sample word once and gathers that word
// from each staged row the cohort keeps (row_of[j] >= 0), repacked and written exactly
// as bed_gather_kernel writes it (padding samples coded 11).
constexpr int kGatherRowsMax = 4;
constexpr int kGatherThreads = 1024;  // one block of four staged rows per SM: 32 warps

__global__ void __launch_bounds__(kGatherThreads)
    bed_gather_cohorts_kernel(const uint8_t* __restrict__ bed, int64_t bpm, int64_t j0,
                              int64_t n_rows, int rpb, const int32_t* __restrict__ sidx,
                              const CohortSet set) {
  extern __shared__ __align__(16) uint8_t row_s[];
  const int64_t stride = (bpm + 31) / 16 * 16;  // round_up(bpm + 16, 16)
  const int64_t jb = j0 + (int64_t)blockIdx.x * rpb;
  const int64_t left = j0 + n_rows - jb;
  const int nr = left < rpb ? (int)left : rpb;
  const uint8_t* src[kGatherRowsMax];
#pragma unroll
  for (int q = 0; q < kGatherRowsMax; ++q)
    src[q] = q < nr ? stage_row(bed + 3 + (jb + q) * bpm, bpm, row_s + q * stride) : nullptr;
  for (int c = 0; c < set.n; ++c) {
    const CohortRows& cr = set.c[c];
    int32_t r[kGatherRowsMax];
    bool any = false;
#pragma unroll
    for (int q = 0; q < kGatherRowsMax; ++q) {
      r[q] = q < nr ? cr.row_of[(jb + q) * cr.row_stride] : -1;
      any |= r[q] >= 0;
    }
    if (!any) continue;
    const int32_t* sc = sidx + cr.sidx_off;
    const bool vec = (reinterpret_cast<uintptr_t>(sc) & 15u) == 0;
    const int64_t n_real = (cr.n + 15) / 16;
    for (int64_t w = threadIdx.x; w < cr.wpr; w += blockDim.x) {
      if (w >= n_real) {
#pragma unroll
        for (int q = 0; q < kGatherRowsMax; ++q)
          if (r[q] >= 0) cr.geno[(int64_t)r[q] * cr.wpr + w] = 0xFFFFFFFFu;
        continue;
      }
      const int64_t k0 = 16 * w;
      const int kn = (cr.n - k0) < 16 ? (int)(cr.n - k0) : 16;
      int32_t ss[16];
      if (vec && kn == 16) {
        const int4* s4 = reinterpret_cast<const int4*>(sc + k0);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          const int4 v = __ldg(s4 + g);
          ss[4 * g] = v.x;
          ss[4 * g + 1] = v.y;
          ss[4 * g + 2] = v.z;
          ss[4 * g + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int e = 0; e < 16; ++e) ss[e] = e < kn ? sc[k0 + e] : 0;
      }
      const uint32_t keep = kn >= 16 ? 0xFFFFFFFFu : ((1u << (2 * kn)) - 1u);
#pragma unroll
      for (int q = 0; q < kGatherRowsMax; ++q) {
        if (r[q] < 0) continue;
        uint32_t word = 0;
#pragma unroll
        for (int e = 0; e < 16; ++e)
          word |= ((uint32_t)(src[q][ss[e] >> 2] >> ((ss[e] & 3) * 2)) & 3u) << (2 * e);
        cr.geno[(int64_t)r[q] * cr.wpr + w] = to_device_layout((word & keep) | ~keep);
      }
    }
  }
}

}  // namespace

cudaError_t launch_bed_gather_cohorts(const uint8_t* bed, int64_t bpm, int64_t j0, int64_t n_rows,
                                      const int32_t* sidx, const CohortSet& set,
                                      cudaStream_t st) {
  if (n_rows <= 0 || set.n <= 0) return cudaSuccess;
  if (set.n > kCohortsPerLaunch) return cudaErrorInvalidValue;
  if (bpm > kSmemRowMax) return cudaErrorInvalidValue;
  // as many rows per block as 200 KB of shared memory hold (each index load then serves
  // all of them), at most kGatherRowsMax
  const int64_t stride = round_up(bpm + 16, 16);
  const int rpb = (int)std::max<int64_t>(1, std::min<int64_t>(kGatherRowsMax, kSmemRowMax / stride));
  const size_t smem = (size_t)(stride * rpb);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(bed_gather_cohorts_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  bed_gather_cohorts_kernel<<<(unsigned)ceil_div(n_rows, rpb), kGatherThreads, smem, st>>>(
      bed, bpm, j0, n_rows, rpb, sidx, set);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_bed_count_cohorts(const uint8_t* bed, int64_t bpm, int64_t j0, int64_t n_rows,
                                     const int32_t* sidx, const int64_t* offs, const int64_t* ns,
                                     int n_cohorts, int64_t m_tot, long long* counts,
                                     cudaStream_t st) {
  if (n_rows <= 0) return cudaSuccess;
  if (bpm > kSmemRowMax) return cudaErrorInvalidValue;  // rows must fit in shared memory
  const size_t smem = (size_t)round_up(bpm + 16, 16);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(bed_count_cohorts_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  bed_count_cohorts_kernel<<<(unsigned)n_rows, kThreads, smem, st>>>(bed, bpm, j0, sidx, offs, ns,
                                                                    n_cohorts, m_tot, counts);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_bed_gather(const uint8_t* bed, int64_t bpm, const int64_t* src_rows,
                              int64_t n_rows, const int32_t* sample_idx, int64_t n,
                              uint32_t* geno_out, int64_t words_per_row, int64_t* counts,
                              cudaStream_t st) {
  if (n_rows <= 0) return cudaSuccess;
  const int use_smem = bpm <= kSmemRowMax ? 1 : 0;
  const size_t smem = use_smem ? (size_t)round_up(bpm + 16, 16) : 0;
  if (sample_idx) {
    auto k = bed_gather_kernel<false>;
    if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    k<<<(unsigned)n_rows, kThreads, smem, st>>>(bed, bpm, src_rows, sample_idx, n, geno_out,
                                                words_per_row, counts, use_smem);
  } else {
    // identity subset: no staging needed, bytes are read in order
    bed_gather_kernel<true><<<(unsigned)n_rows, kThreads, 0, st>>>(
        bed, bpm, src_rows, nullptr, n, geno_out, words_per_row, counts, 0);
  }
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace saige
