// Missing-call lists for the one-column products (see miss_lists.cuh).
//
// A one-column MIXED product forms, per marker (pass A) or per sample (pass B), the
// integer sums G = sum g q over the calls and Mi = sum q over the missing calls
// (kernels_tc.cu).  With ~1 % of calls missing, the dense missing-flag sums cost a
// third of the kernels' instructions (one byte permute and three dp4a per four
// entries) for a sum over a few entries.  With these lists the one-column kernels form
// Mi instead as an exact int64 sum of the quantised vector over each row's missing
// calls, read from the chunk of the vector they already hold in shared memory.  The
// integer is the one the dense sums form, so the products do not change by a bit.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "miss_lists.cuh"

namespace saige {

namespace {

constexpr int kTileRows = 128;        // rows of a sample-major code tile
constexpr int64_t kTileBytes = 4096;  // 128 rows x 128 entries x 2 bits

// The missing calls (code 01: low bit set, high bit clear) of a packed word, as its
// even bits.
__device__ __forceinline__ uint32_t missing_bits(uint32_t w) {
  return w & ~(w >> 1) & 0x55555555u;
}

// Flagged bits of a device-layout word (entry 4j + i at bit 16(j>>1) + 2(j&1) + 4i) as
// a 16-bit mask in entry order: bit c/2 = 8(j>>1) + (j&1) + 2i gives j = 2(c>>3) + (c&1)
// and i = (c>>1) & 3.
__device__ __forceinline__ uint32_t entry_order(uint32_t bits) {
  uint32_t e = 0;
  while (bits) {
    const int c = (__ffs(bits) - 1) >> 1;
    bits &= bits - 1;
    e |= 1u << (4 * (2 * (c >> 3) + (c & 1)) + ((c >> 1) & 3));
  }
  return e;
}

// Writes tag | (base + e) for the set bits e of mask, ascending, at ent[pos...].
__device__ __forceinline__ void emit(uint32_t mask, uint32_t tag, uint32_t base, uint32_t* ent,
                                     int64_t& pos) {
  while (mask) {
    const int e = __ffs(mask) - 1;
    mask &= mask - 1;
    ent[pos++] = tag | (base + (uint32_t)e);
  }
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Pass A segments: grid (m_pad / a_rows, nch), block 256 (8 warps, a_rows / 8 rows
// each); block (b, c) takes words [c cw, (c + 1) cw) of its rows.  Counting writes the
// segment's size; filling writes its entries ordered by row, then sample (per-row
// counts, a scan over the block's rows, then a warp prefix sum over each round of 32
// words).
template <bool kFill>
__global__ void __launch_bounds__(256)
    miss_a_kernel(const uint32_t* __restrict__ geno, int64_t wpr, int a_rows, int64_t cw,
                  int64_t nch, int bits, int32_t* __restrict__ seg_cnt,
                  const int64_t* __restrict__ seg, uint32_t* __restrict__ ent) {
  __shared__ int rc[256];
  __shared__ int64_t rstart[256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int per_warp = a_rows / 8;
  const int64_t b = blockIdx.x, c = blockIdx.y;
  const int64_t w0 = c * cw, w1 = w0 + cw < wpr ? w0 + cw : wpr;
  for (int k = 0; k < per_warp; ++k) {
    const uint32_t* r = geno + (b * a_rows + warp * per_warp + k) * wpr;
    int n = 0;
    for (int64_t t = w0 + lane; t < w1; t += 32) n += __popc(missing_bits(__ldg(r + t)));
    n = warp_sum(n);
    if (lane == 0) rc[warp * per_warp + k] = n;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t p = kFill ? seg[b * nch + c] : 0;
    for (int i = 0; i < a_rows; ++i) {
      rstart[i] = p;
      p += rc[i];
    }
    if (!kFill) seg_cnt[b * nch + c] = (int32_t)p;
  }
  if (!kFill) return;
  __syncthreads();
  for (int k = 0; k < per_warp; ++k) {
    const int rb = warp * per_warp + k;
    const uint32_t* r = geno + (b * a_rows + rb) * wpr;
    int64_t pos = rstart[rb];
    for (int64_t t0 = w0; t0 < w1; t0 += 32) {
      const int64_t t = t0 + lane;
      const uint32_t mis = t < w1 ? missing_bits(__ldg(r + t)) : 0u;
      const int n = __popc(mis);
      int incl = n;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (n) {
        int64_t q = pos + incl - n;
        emit(entry_order(mis), (uint32_t)rb << bits, (uint32_t)(16 * (t - w0)), ent, q);
      }
      pos += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
}

// Pass B segments: grid (n_pad / 256, nch), block 256, thread = sample h 128 + r of the
// sample tiles 2p, 2p + 1 (h = thread / 128); block (p, c) takes the marker tiles of
// chunk c (ct = chunk / 128 of them).  Counting writes the segment's size; filling writes
// its entries ordered by sample, then marker (a scan over the block's threads).
template <bool kFill>
__global__ void __launch_bounds__(256)
    miss_b_kernel(const uint8_t* __restrict__ tiles_s, int64_t s_ld, int64_t n_mt, int64_t ct,
                  int64_t nch, int bits, int32_t* __restrict__ seg_cnt,
                  const int64_t* __restrict__ seg, uint32_t* __restrict__ ent) {
  __shared__ int tc[256];
  __shared__ int64_t tstart[256];
  const int tid = threadIdx.x;
  const int64_t p = blockIdx.x, c = blockIdx.y;
  const int64_t st = 2 * p + (tid >> 7);
  const int r = tid & 127;
  const int64_t mt0 = c * ct, mt1 = mt0 + ct < n_mt ? mt0 + ct : n_mt;
  auto words = [&](int64_t mt, uint32_t w[8]) {
    const uint4* row =
        reinterpret_cast<const uint4*>(tiles_s + (st * s_ld + mt) * kTileBytes + (int64_t)r * 32);
    const uint4 h0 = __ldg(row), h1 = __ldg(row + 1);
    w[0] = h0.x; w[1] = h0.y; w[2] = h0.z; w[3] = h0.w;
    w[4] = h1.x; w[5] = h1.y; w[6] = h1.z; w[7] = h1.w;
  };
  int n = 0;
  for (int64_t mt = mt0; mt < mt1; ++mt) {
    uint32_t w[8];
    words(mt, w);
#pragma unroll
    for (int j = 0; j < 8; ++j) n += __popc(missing_bits(w[j]));
  }
  tc[tid] = n;
  __syncthreads();
  if (tid == 0) {
    int64_t q = kFill ? seg[p * nch + c] : 0;
    for (int i = 0; i < 256; ++i) {
      tstart[i] = q;
      q += tc[i];
    }
    if (!kFill) seg_cnt[p * nch + c] = (int32_t)q;
  }
  if (!kFill) return;
  __syncthreads();
  int64_t pos = tstart[tid];
  for (int64_t mt = mt0; mt < mt1; ++mt) {
    uint32_t w[8];
    words(mt, w);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t mis = missing_bits(w[j]);
      if (mis)
        emit(entry_order(mis), (uint32_t)tid << bits,
             (uint32_t)((mt - mt0) * kTileRows + 16 * j), ent, pos);
    }
  }
}

int log2_exact(int64_t x) {
  int b = 0;
  while ((int64_t(1) << b) < x) ++b;
  return (int64_t(1) << b) == x ? b : -1;
}

// Exclusive scan of n counts into n + 1 offsets.
std::vector<int64_t> offsets(const int32_t* cnt, int64_t n) {
  std::vector<int64_t> o((size_t)n + 1, 0);
  for (int64_t i = 0; i < n; ++i) o[(size_t)i + 1] = o[(size_t)i] + cnt[i];
  return o;
}

}  // namespace

Status miss_lists_build(saige_grm* h, const uint8_t* tiles_s, int64_t s_ld, const MissShape& sh,
                        MissLists* L, cudaStream_t st) {
  L->state = -1;
  const int64_t m_pad = h->m_pad, n_pad = h->n_pad, n_mt = m_pad / kTileRows;
  const int a_bits = log2_exact(16 * sh.a_chunk_words), b_bits = log2_exact(sh.b_chunk);
  if (sh.a_rows % 8 || sh.a_rows > 256 || m_pad % sh.a_rows || log2_exact(sh.a_rows) < 0 ||
      a_bits < 0 || a_bits + log2_exact(sh.a_rows) > 32 || sh.b_rows != 2 * kTileRows ||
      n_pad % sh.b_rows || b_bits < 0 || sh.b_chunk % kTileRows || b_bits + 8 > 32)
    return fail(SAIGE_EINVAL, "missing-call lists: unsupported kernel shape");
  const int64_t nba = m_pad / sh.a_rows, ncha = ceil_div(h->wpr, sh.a_chunk_words);
  const int64_t nbb = n_pad / sh.b_rows, ct = sh.b_chunk / kTileRows, nchb = ceil_div(n_mt, ct);
  DevBuf cnt;
  if (!cnt.reserve((size_t)(nba * ncha + nbb * nchb) * sizeof(int32_t)).ok()) return Status();
  int32_t* ca = cnt.as<int32_t>();
  int32_t* cb = ca + nba * ncha;
  miss_a_kernel<false><<<dim3((unsigned)nba, (unsigned)ncha), 256, 0, st>>>(
      h->geno, h->wpr, sh.a_rows, sh.a_chunk_words, ncha, a_bits, ca, nullptr, nullptr);
  miss_b_kernel<false><<<dim3((unsigned)nbb, (unsigned)nchb), 256, 0, st>>>(
      tiles_s, s_ld, n_mt, ct, nchb, b_bits, cb, nullptr, nullptr);
  SG_CHECK_LAUNCH();
  count_launches(2);
  std::vector<int32_t> hc((size_t)(nba * ncha + nbb * nchb));
  SG_CUDA(cudaMemcpyAsync(hc.data(), ca, hc.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  const std::vector<int64_t> oa = offsets(hc.data(), nba * ncha);
  const std::vector<int64_t> ob = offsets(hc.data() + nba * ncha, nbb * nchb);
  const int64_t total = oa.back();
  if (ob.back() != total)
    return fail(SAIGE_ECUDA, "missing-call lists: %lld calls by marker, %lld by sample",
                (long long)total, (long long)ob.back());
  if ((double)total > kMissListMaxFrac * (double)h->m * (double)h->n) return Status();
  const size_t ent_bytes = (size_t)std::max<int64_t>(total, 1) * sizeof(uint32_t);
  // the lists are optional: declined rather than have an allocation flush the block cache
  // (freeing every cached block) when the free memory would not hold them with room over
  size_t free_b = 0, total_b = 0;
  SG_CUDA(cudaMemGetInfo(&free_b, &total_b));
  if (free_b < 2 * ent_bytes + ((size_t)1 << 30)) return Status();
  if (!L->a_seg.reserve(oa.size() * sizeof(int64_t)).ok() ||
      !L->b_seg.reserve(ob.size() * sizeof(int64_t)).ok() || !L->a_ent.reserve(ent_bytes).ok() ||
      !L->b_ent.reserve(ent_bytes).ok()) {
    L->a_seg.release();
    L->b_seg.release();
    L->a_ent.release();
    L->b_ent.release();
    return Status();
  }
  SG_CUDA(cudaMemcpyAsync(L->a_seg.ptr, oa.data(), oa.size() * sizeof(int64_t),
                          cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemcpyAsync(L->b_seg.ptr, ob.data(), ob.size() * sizeof(int64_t),
                          cudaMemcpyHostToDevice, st));
  miss_a_kernel<true><<<dim3((unsigned)nba, (unsigned)ncha), 256, 0, st>>>(
      h->geno, h->wpr, sh.a_rows, sh.a_chunk_words, ncha, a_bits, nullptr,
      L->a_seg.as<int64_t>(), L->a_ent.as<uint32_t>());
  miss_b_kernel<true><<<dim3((unsigned)nbb, (unsigned)nchb), 256, 0, st>>>(
      tiles_s, s_ld, n_mt, ct, nchb, b_bits, nullptr, L->b_seg.as<int64_t>(),
      L->b_ent.as<uint32_t>());
  SG_CHECK_LAUNCH();
  count_launches(2);
  // the segment offsets are read from oa and ob until the copies are done
  SG_CUDA(cudaStreamSynchronize(st));
  L->a_nch = ncha;
  L->b_nch = nchb;
  L->a_bits = a_bits;
  L->b_bits = b_bits;
  L->total = total;
  L->state = 1;
  return Status();
}

}  // namespace saige
