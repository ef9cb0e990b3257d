// MIXED-precision GRM product on the 5th-generation tensor cores.
//
//   pass A  u[m,r] = (1/s_m) sum_i nm_mi (g_mi - 2p_m) v[i,r]
//   pass B  y[i,r] = (1/M)   sum_m nm_mi (g_mi - 2p_m) u[m,r] / s_m
//
// which is OnTheFlyGrm::mat_vec (saige-core/src/glmm/pcg.rs:128-180) with the
// standardisation of OnTheFlyGrm::new (pcg.rs:101-122) folded into the
// product and missing calls centred to zero, without materialising Z.
//
// Arithmetic.  Each column of v (pass A) and of w = u/s, c = 2p w (pass B) is
// quantised to a signed integer q with |q| <= 127*2^16 (24 bits) and split
// into three signed int8 limbs q = 2^16 l2 + 2^8 l1 + l0.  Genotypes
// g in {0,1,2} and the missing indicator are exact int8 operands.
// tcgen05.mma kind::i8 accumulates exact s32 sums per limb in TMEM; limbs,
// scales and the per-marker 2p, 1/s are combined in FP64 in the epilogue:
//   sum_i nm (g - 2p) v = scale (G - 2p (S - Mi)),  G = sum g q, Mi = sum miss q,
//   S = sum q (exact int64), so the only error is the rounding of v to q.
//
// Data movement.  The packed 2-bit rows (HBM, 128-byte aligned) arrive by TMA
// (2D tensor map, 128 rows x 32 bytes = 128 samples per stage); the quantised
// vector operand arrives by one bulk copy per stage from an image written
// already in the swizzled shared-memory layout.  Four warps expand the 2-bit
// codes into the two int8 operand tiles with byte permutes (PRMT) and write
// them in the 128-byte-swizzled layout the MMA reads:
//   pass A: rows = markers (M), 128 samples = K  -> K-major A
//   pass B: rows = markers (K), 128 samples = M  -> MN-major A
// Roles: warp 0 issues TMA, warp 1 owns TMEM and issues MMAs, warps 2-5 unpack
// and then run the epilogue.  Every mbarrier wait is bounded; a wait that runs
// out sets an error word the host reads back (SAIGE_TIMEOUT).
#include <cuda.h>
#include <math.h>

#include <vector>

#include "kernels.cuh"
#include "kernels_tc.cuh"

namespace saige {

namespace {

constexpr int kRows = 128;     // MMA M: rows of a CTA tile
constexpr int kKt = 128;       // K per pipeline stage
constexpr int kStages = 2;
constexpr int kThreads = 192;  // 6 warps
constexpr int kMaxR = 64;      // right-hand sides per launch (3*64 = 192 <= 256 MMA N)
constexpr double kQ = 127.0 * 65536.0;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

struct TcArgs {
  int ng;                   // B tile rows (= MMA N), multiple of 16
  int r;                    // right-hand sides in this launch
  int nk;                   // pipeline stages over K
  const uint8_t* img_g;     // nk x ng x 128 bytes
  const uint8_t* img_m;     // pass B: c image (same shape); pass A: unused
  const double* scale_g;    // [r]
  const double* scale_m;    // [r] pass B
  const long long* sum_q;   // [r] pass A: sum q_v; pass B: sum q_c
  const double* two_p;      // [m_pad]
  const double* inv_s;      // [m_pad]
  double* out;              // pass A: u [r][out_ld]; pass B: kp (column col_map[r])
  int64_t out_ld;
  const int* col_map;       // pass B
  double out_scale;         // pass B: 1/M
  unsigned int* err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false (and raises the CTA abort flag and the error
// word) when the barrier phase does not complete in time or another role
// already gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned int* err) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > kWaitCycles) {
      *abort_flag = 1;
      atomicOr(err, 1u);
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Shared-memory matrix descriptor, 128-byte swizzle, version 1 (sm_100).
// K-major:  SBO = 1024 B between 8-row groups, LBO unused (1).
// MN-major: SBO = 1024 B between 8-row K groups, one 128-byte atom along M.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr, bool mn_major) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)(mn_major ? 64u : 1u) << 16;   // leading byte offset >> 4
  d |= (uint64_t)64u << 32;                      // stride byte offset (1024) >> 4
  d |= (uint64_t)1u << 46;                       // version
  d |= (uint64_t)2u << 61;                       // SWIZZLE_128B
  return d;
}

// Instruction descriptor: kind::i8, s32 accumulate, signed A and B, M = 128.
__host__ __device__ constexpr uint32_t i8_idesc(int n, bool a_mn_major) {
  return (2u << 4)                        // c_format = S32
         | (1u << 7)                      // a_format = signed int8
         | (1u << 10)                     // b_format = signed int8
         | ((a_mn_major ? 1u : 0u) << 15) // a_major
         | (0u << 16)                     // b_major = K
         | ((uint32_t)(n >> 3) << 17)     // N >> 3
         | ((uint32_t)(kRows >> 4) << 24);// M >> 4
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Spread the 8 codes of bytes (b_lo, b_hi) of w into two 16-bit PRMT selectors
// (one nibble per code).  sel = PRMT(w, 0, 0x4140 | ...) puts byte b_lo in
// bits 0-7 and byte b_hi in bits 16-23, then nibble- and 2-bit-spreading.
__device__ __forceinline__ uint32_t spread_pair(uint32_t w, uint32_t prmt_sel) {
  uint32_t t = __byte_perm(w, 0u, prmt_sel);
  t = (t | (t << 4)) & 0x0F0F0F0Fu;
  t = (t | (t << 2)) & 0x33333333u;
  return t;
}

// Codes 00,01,10,11 -> genotype bytes {2,0,1,0} and missing bytes {0,1,0,0}.
constexpr uint32_t kLutG = 0x00010002u;
constexpr uint32_t kLutM = 0x00000100u;

template <bool kPassB>
__global__ void __launch_bounds__(kThreads, 1)
    tc_grm_kernel(const __grid_constant__ CUtensorMap codes_map, TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  // carve 1024-aligned regions
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* sbase = smem_raw + (base - raw);
  const uint32_t a_bytes = kRows * kKt;                  // 16 KB per int8 tile
  const uint32_t b_bytes = (uint32_t)a.ng * kKt;         // ng x 128 B
  const uint32_t nb = kPassB ? 2u : 1u;
  const uint32_t stage_bytes = 2u * a_bytes + nb * b_bytes + kRows * 32u;
  auto A_g = [&](int s) { return base + (uint32_t)s * stage_bytes; };
  auto A_m = [&](int s) { return A_g(s) + a_bytes; };
  auto B_g = [&](int s) { return A_g(s) + 2u * a_bytes; };
  auto B_m = [&](int s) { return B_g(s) + b_bytes; };
  auto CODES = [&](int s) { return A_g(s) + 2u * a_bytes + nb * b_bytes; };
  const uint32_t bar_base = base + kStages * stage_bytes;
  auto FULL = [&](int s) { return bar_base + 8u * s; };
  auto UNP = [&](int s) { return bar_base + 8u * (kStages + s); };
  auto EMPTY = [&](int s) { return bar_base + 8u * (2 * kStages + s); };
  const uint32_t ACCF = bar_base + 8u * (3 * kStages);
  uint8_t* misc = sbase + (bar_base - base) + 8u * (3 * kStages + 1);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(misc);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(misc + 8);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const uint32_t tmem_cols_needed = 2u * a.ng;
  uint32_t tmem_cols = 32;
  while (tmem_cols < tmem_cols_needed) tmem_cols <<= 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(FULL(s), 1);
      mbar_init(UNP(s), 128);
      mbar_init(EMPTY(s), 1);
    }
    mbar_init(ACCF, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t tmem_g = tmem, tmem_m = tmem + (uint32_t)a.ng;

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      const uint32_t tx = kRows * 32u + nb * b_bytes;
      for (int k = 0; k < a.nk; ++k) {
        const int s = k % kStages;
        if (k >= kStages && !mbar_wait(EMPTY(s), (uint32_t)((k / kStages) - 1) & 1u, abort_flag, a.err))
          break;
        mbar_expect_tx(FULL(s), tx);
        // pass A: x = 32-byte column of samples k, y = marker tile;
        // pass B: x = sample tile, y = marker block k.
        const int x = kPassB ? tile * 32 : k * 32;
        const int y = kPassB ? k * kRows : tile * kRows;
        tma_load_2d(CODES(s), &codes_map, x, y, FULL(s));
        bulk_load(B_g(s), a.img_g + (size_t)k * b_bytes, b_bytes, FULL(s));
        if (kPassB) bulk_load(B_m(s), a.img_m + (size_t)k * b_bytes, b_bytes, FULL(s));
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = i8_idesc(a.ng, kPassB);
      bool ok = true;
      for (int k = 0; k < a.nk && ok; ++k) {
        const int s = k % kStages;
        if (!mbar_wait(UNP(s), (uint32_t)(k / kStages) & 1u, abort_flag, a.err)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t ag = sw128_desc(A_g(s), kPassB), am = sw128_desc(A_m(s), kPassB);
        const uint64_t bg = sw128_desc(B_g(s), false);
        const uint64_t bm = sw128_desc(kPassB ? B_m(s) : B_g(s), false);
#pragma unroll
        for (int kk = 0; kk < kKt / 32; ++kk) {
          // K advance of 32: 32 bytes along a K-major row, or 32 rows (4 KB) of an MN-major tile
          const uint64_t da = kPassB ? (uint64_t)(kk * 256) : (uint64_t)(kk * 2);
          const uint64_t db = (uint64_t)(kk * 2);
          const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
          mma_i8(tmem_g, ag + da, bg + db, idesc, acc);
          mma_i8(tmem_m, am + da, bm + db, idesc, acc);
        }
        mma_commit(EMPTY(s));
      }
      mma_commit(ACCF);
    }
  } else {
    // ---------------- unpack (warps 2-5) ----------------
    const int row = threadIdx.x - 64;  // code row 0..127
    uint8_t* smem_gen = sbase;
    for (int k = 0; k < a.nk; ++k) {
      const int s = k % kStages;
      if (!mbar_wait(FULL(s), (uint32_t)(k / kStages) & 1u, abort_flag, a.err)) break;
      const uint4* crow = reinterpret_cast<const uint4*>(smem_gen + (CODES(s) - base) + row * 32);
      const uint4 c0 = crow[0], c1 = crow[1];
      const uint32_t words[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
      uint8_t* ag = smem_gen + (A_g(s) - base) + row * 128;
      uint8_t* am = smem_gen + (A_m(s) - base) + row * 128;
      const int sw = row & 7;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const uint32_t w = words[c];
        const uint32_t s01 = spread_pair(w, 0x4140u);
        const uint32_t s23 = spread_pair(w, 0x4342u);
        uint4 g, m;
        g.x = __byte_perm(kLutG, 0u, s01);
        g.y = __byte_perm(kLutG, 0u, s01 >> 16);
        g.z = __byte_perm(kLutG, 0u, s23);
        g.w = __byte_perm(kLutG, 0u, s23 >> 16);
        m.x = __byte_perm(kLutM, 0u, s01);
        m.y = __byte_perm(kLutM, 0u, s01 >> 16);
        m.z = __byte_perm(kLutM, 0u, s23);
        m.w = __byte_perm(kLutM, 0u, s23 >> 16);
        const int pos = (c ^ sw) * 16;
        *reinterpret_cast<uint4*>(ag + pos) = g;
        *reinterpret_cast<uint4*>(am + pos) = m;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(UNP(s));
    }
    // ---------------- epilogue ----------------
    __syncwarp();
    const int lg = warp & 3;  // TMEM lane group this warp may access
    const int trow = lg * 32 + lane;
    const bool ok = mbar_wait(ACCF, 0u, abort_flag, a.err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t grow = (int64_t)tile * kRows + trow;  // marker (A) or sample (B)
    double rowa = 0.0, rowb = 0.0;
    if (!kPassB) {
      rowa = a.inv_s[grow];
      rowb = a.two_p[grow];
    }
    for (int r0 = 0; r0 < a.r; r0 += 16) {
      uint32_t g[48], m[48];
      const uint32_t lane_off = (uint32_t)(lg * 32) << 16;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int col = 3 * r0 + 16 * j;
        if (col < a.ng) {
          uint32_t t[16];
          tmem_ld16(tmem_g + lane_off + (uint32_t)col, t);
#pragma unroll
          for (int e = 0; e < 16; ++e) g[16 * j + e] = t[e];
          tmem_ld16(tmem_m + lane_off + (uint32_t)col, t);
#pragma unroll
          for (int e = 0; e < 16; ++e) m[16 * j + e] = t[e];
        }
      }
      tmem_wait_ld();
      if (!ok) continue;
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int r = r0 + e;
        if (r >= a.r) break;
        const double G = 65536.0 * (double)(int)g[3 * e] + 256.0 * (double)(int)g[3 * e + 1] +
                         (double)(int)g[3 * e + 2];
        const double Mi = 65536.0 * (double)(int)m[3 * e] + 256.0 * (double)(int)m[3 * e + 1] +
                          (double)(int)m[3 * e + 2];
        const double S = (double)a.sum_q[r];
        if (!kPassB) {
          // u = (1/s) scale (G - 2p (S - Mi)); explicit roundings (no contraction)
          const double t = __dsub_rn(G, __dmul_rn(rowb, S - Mi));
          a.out[(int64_t)r * a.out_ld + grow] = __dmul_rn(rowa, __dmul_rn(a.scale_g[r], t));
        } else {
          // y = (1/M) (sw G - sc (S_c - Mc))
          const double y = __dmul_rn(a.out_scale, __dsub_rn(__dmul_rn(a.scale_g[r], G),
                                                            __dmul_rn(a.scale_m[r], S - Mi)));
          a.out[(int64_t)a.col_map[r] * a.out_ld + grow] = y;
        }
      }
    }
  }

  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(tmem_cols));
  }
}

// ---------------------------------------------------------------------------
// quantisation kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v) {
  atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// amax over rows [0, len) of column col_map[r] (pass A input v)
__global__ void amax_v_kernel(const double* __restrict__ v, int64_t ld, int64_t len,
                              const int* __restrict__ col_map, unsigned long long* amax) {
  const int r = blockIdx.y;
  const double* c = v + (int64_t)col_map[r] * ld;
  double m = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(c[i]));
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomic_max_nonneg(&amax[r], m);
}

// amax of w = u inv_s and c = w 2p over markers
__global__ void amax_wc_kernel(const double* __restrict__ u, int64_t ld, int64_t len,
                               const double* __restrict__ inv_s, const double* __restrict__ two_p,
                               unsigned long long* amax_w, unsigned long long* amax_c) {
  const int r = blockIdx.y;
  const double* c = u + (int64_t)r * ld;
  double mw = 0.0, mc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double w = c[i] * inv_s[i];
    mw = fmax(mw, fabs(w));
    mc = fmax(mc, fabs(w * two_p[i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mw = fmax(mw, __shfl_xor_sync(0xffffffffu, mw, o));
    mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, o));
  }
  if ((threadIdx.x & 31) == 0) {
    if (mw > 0.0) atomic_max_nonneg(&amax_w[r], mw);
    if (mc > 0.0) atomic_max_nonneg(&amax_c[r], mc);
  }
}

__device__ __forceinline__ double scale_of(unsigned long long bits) {
  const double amax = __longlong_as_double((long long)bits);
  return amax > 0.0 ? amax / kQ : 1.0;
}

// Split q (|q| <= 127*2^16) into signed limbs q = 2^16 l2 + 2^8 l1 + l0.
__device__ __forceinline__ void limbs(long long q, int& l2, int& l1, int& l0) {
  l0 = (int)(signed char)(q & 0xFF);
  const long long q1 = (q - l0) >> 8;
  l1 = (int)(signed char)(q1 & 0xFF);
  l2 = (int)((q1 - l1) >> 8);
}

__device__ __forceinline__ void put_limbs(uint8_t* stage_img, int r, int pos, long long q) {
  int l2, l1, l0;
  limbs(q, l2, l1, l0);
  const int rows[3] = {3 * r, 3 * r + 1, 3 * r + 2};
  const int vals[3] = {l2, l1, l0};
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const int row = rows[j];
    const int off = row * 128 + (((pos >> 4) ^ (row & 7)) << 4) + (pos & 15);
    stage_img[off] = (uint8_t)(signed char)vals[j];
  }
}

__device__ __forceinline__ long long block_sum_ll(long long v, long long* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  long long s = 0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
  return s;
}

// One block = one 128-row stage of one column: quantise v, write the limbs
// into the swizzled stage image, accumulate sum q.
__global__ void __launch_bounds__(128)
    quant_v_kernel(const double* __restrict__ v, int64_t ld, int64_t len,
                   const int* __restrict__ col_map, const unsigned long long* __restrict__ amax,
                   double* __restrict__ scale_out, uint8_t* __restrict__ img, int ng,
                   unsigned long long* __restrict__ sum_q) {
  __shared__ long long sh[4];
  const int r = blockIdx.y;
  const int64_t stage = blockIdx.x;
  const int pos = threadIdx.x;
  const int64_t i = stage * 128 + pos;
  const double sc = scale_of(amax[r]);
  const double x = i < len ? v[(int64_t)col_map[r] * ld + i] : 0.0;
  const long long q = __double2ll_rn(x / sc);
  put_limbs(img + stage * (int64_t)ng * 128, r, pos, q);
  const long long s = block_sum_ll(q, sh);
  if (threadIdx.x == 0) {
    atomicAdd(&sum_q[r], (unsigned long long)s);
    if (stage == 0) scale_out[r] = sc;
  }
}

__global__ void __launch_bounds__(128)
    quant_wc_kernel(const double* __restrict__ u, int64_t ld, const double* __restrict__ inv_s,
                    const double* __restrict__ two_p, const unsigned long long* __restrict__ amax_w,
                    const unsigned long long* __restrict__ amax_c, double* __restrict__ scale_w,
                    double* __restrict__ scale_c, uint8_t* __restrict__ img_w,
                    uint8_t* __restrict__ img_c, int ng, unsigned long long* __restrict__ sum_c) {
  __shared__ long long sh[4];
  const int r = blockIdx.y;
  const int64_t stage = blockIdx.x;
  const int pos = threadIdx.x;
  const int64_t m = stage * 128 + pos;
  const double sw = scale_of(amax_w[r]), scc = scale_of(amax_c[r]);
  const double w = u[(int64_t)r * ld + m] * inv_s[m];
  const double c = w * two_p[m];
  const long long qw = __double2ll_rn(w / sw);
  const long long qc = __double2ll_rn(c / scc);
  put_limbs(img_w + stage * (int64_t)ng * 128, r, pos, qw);
  put_limbs(img_c + stage * (int64_t)ng * 128, r, pos, qc);
  const long long s = block_sum_ll(qc, sh);
  if (threadIdx.x == 0) {
    atomicAdd(&sum_c[r], (unsigned long long)s);
    if (stage == 0) {
      scale_w[r] = sw;
      scale_c[r] = scc;
    }
  }
}

size_t tc_smem_bytes(int ng, bool pass_b) {
  const size_t a_bytes = (size_t)kRows * kKt;
  const size_t b_bytes = (size_t)ng * kKt;
  const size_t stage = 2 * a_bytes + (pass_b ? 2 : 1) * b_bytes + kRows * 32;
  return 1024 + kStages * stage + 8 * (3 * kStages + 1) + 16;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

struct TcPlan {
  CUtensorMap codes_map;
  DevBuf img_a, img_w, img_c, u, scal, cmap;
  int cap_r = 0;
};

static Status tc_init(saige_grm* h) {
  if (h->tc) return Status();
  TcPlan* p = new TcPlan();
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  SG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (!fn || q != cudaDriverEntryPointSuccess) {
    delete p;
    return fail(SAIGE_ECUDA, "cuTensorMapEncodeTiled is not available");
  }
  const cuuint64_t dims[2] = {(cuuint64_t)(h->wpr * 4), (cuuint64_t)h->m_pad};
  const cuuint64_t strides[1] = {(cuuint64_t)(h->wpr * 4)};
  const cuuint32_t box[2] = {32, (cuuint32_t)kRows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = reinterpret_cast<EncodeTiledFn>(fn)(
      &p->codes_map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)h->geno, dims, strides, box, estr,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    delete p;
    return fail(SAIGE_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  }
  for (auto kern : {tc_grm_kernel<false>, tc_grm_kernel<true>}) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tc_smem_bytes(256, true));
    if (e != cudaSuccess) {
      delete p;
      return fail(SAIGE_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    }
  }
  h->tc = p;
  return Status();
}

void tc_destroy(saige_grm* h) {
  if (!h || !h->tc) return;
  delete h->tc;
  h->tc = nullptr;
}

// Scalar block layout (device): per launch of R <= kMaxR columns.
struct Scal {
  unsigned long long* amax_v;  // R
  unsigned long long* amax_w;
  unsigned long long* amax_c;
  unsigned long long* sum_v;
  unsigned long long* sum_c;
  double* scale_v;
  double* scale_w;
  double* scale_c;
  unsigned int* err;
};

static Scal carve(TcPlan* p) {
  char* b = p->scal.as<char>();
  Scal s;
  s.amax_v = reinterpret_cast<unsigned long long*>(b);
  s.amax_w = s.amax_v + kMaxR;
  s.amax_c = s.amax_w + kMaxR;
  s.sum_v = s.amax_c + kMaxR;
  s.sum_c = s.sum_v + kMaxR;
  s.scale_v = reinterpret_cast<double*>(s.sum_c + kMaxR);
  s.scale_w = s.scale_v + kMaxR;
  s.scale_c = s.scale_w + kMaxR;
  s.err = reinterpret_cast<unsigned int*>(s.scale_c + kMaxR);
  return s;
}

Status tc_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                  cudaStream_t st) {
  SG_TRY(tc_init(h));
  TcPlan* p = h->tc;
  std::vector<int> cols;
  for (int c = 0; c < q; ++c)
    if (!active || active[c] == kColActive) cols.push_back(c);
  if (cols.empty()) return Status();
  const int64_t n_stages_a = h->n_pad / kKt;  // samples
  const int64_t n_stages_b = h->m_pad / kKt;  // markers
  const int rmax = (int)std::min<size_t>(cols.size(), (size_t)kMaxR);
  const int ng_max = (int)round_up(3 * rmax, 16);
  SG_TRY(p->img_a.reserve((size_t)h->n_pad * ng_max));
  SG_TRY(p->img_w.reserve((size_t)h->m_pad * ng_max));
  SG_TRY(p->img_c.reserve((size_t)h->m_pad * ng_max));
  SG_TRY(p->u.reserve((size_t)h->m_pad * rmax * sizeof(double)));
  SG_TRY(p->scal.reserve(9 * kMaxR * 8 + 64));
  SG_TRY(p->cmap.reserve((size_t)q * sizeof(int) + 64));
  Scal sc = carve(p);
  SG_CUDA(cudaMemcpyAsync(p->cmap.ptr, cols.data(), cols.size() * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(unsigned int), st));
  for (size_t c0 = 0; c0 < cols.size(); c0 += kMaxR) {
    const int r = (int)std::min<size_t>(kMaxR, cols.size() - c0);
    const int ng = (int)round_up(3 * r, 16);
    const int* cmap = p->cmap.as<int>() + c0;
    SG_CUDA(cudaMemsetAsync(p->scal.ptr, 0, 5 * kMaxR * 8, st));
    SG_CUDA(cudaMemsetAsync(p->img_a.ptr, 0, (size_t)h->n_pad * ng, st));
    // ---- pass A operand ----
    {
      dim3 g1((unsigned)std::min<int64_t>(ceil_div(h->n, 256), 296), (unsigned)r);
      amax_v_kernel<<<g1, 256, 0, st>>>(v, h->n_pad, h->n, cmap, sc.amax_v);
      dim3 g2((unsigned)n_stages_a, (unsigned)r);
      quant_v_kernel<<<g2, 128, 0, st>>>(v, h->n_pad, h->n, cmap, sc.amax_v, sc.scale_v,
                                         p->img_a.as<uint8_t>(), ng, sc.sum_v);
      SG_CHECK_LAUNCH();
    }
    // ---- pass A: u = Z' v ----
    {
      TcArgs a{};
      a.ng = ng;
      a.r = r;
      a.nk = (int)n_stages_a;
      a.img_g = p->img_a.as<uint8_t>();
      a.img_m = nullptr;
      a.scale_g = sc.scale_v;
      a.sum_q = reinterpret_cast<const long long*>(sc.sum_v);
      a.two_p = h->two_p;
      a.inv_s = h->inv_s;
      a.out = p->u.as<double>();
      a.out_ld = h->m_pad;
      a.err = sc.err;
      tc_grm_kernel<false><<<(unsigned)(h->m_pad / kRows), kThreads, tc_smem_bytes(ng, false), st>>>(
          p->codes_map, a);
      SG_CHECK_LAUNCH();
    }
    // ---- pass B operands ----
    {
      SG_CUDA(cudaMemsetAsync(p->img_w.ptr, 0, (size_t)h->m_pad * ng, st));
      SG_CUDA(cudaMemsetAsync(p->img_c.ptr, 0, (size_t)h->m_pad * ng, st));
      dim3 g1((unsigned)std::min<int64_t>(ceil_div(h->m_pad, 256), 296), (unsigned)r);
      amax_wc_kernel<<<g1, 256, 0, st>>>(p->u.as<double>(), h->m_pad, h->m_pad, h->inv_s,
                                         h->two_p, sc.amax_w, sc.amax_c);
      dim3 g2((unsigned)n_stages_b, (unsigned)r);
      quant_wc_kernel<<<g2, 128, 0, st>>>(p->u.as<double>(), h->m_pad, h->inv_s, h->two_p,
                                          sc.amax_w, sc.amax_c, sc.scale_w, sc.scale_c,
                                          p->img_w.as<uint8_t>(), p->img_c.as<uint8_t>(), ng,
                                          sc.sum_c);
      SG_CHECK_LAUNCH();
    }
    // ---- pass B: y = Z w / M ----
    {
      TcArgs a{};
      a.ng = ng;
      a.r = r;
      a.nk = (int)n_stages_b;
      a.img_g = p->img_w.as<uint8_t>();
      a.img_m = p->img_c.as<uint8_t>();
      a.scale_g = sc.scale_w;
      a.scale_m = sc.scale_c;
      a.sum_q = reinterpret_cast<const long long*>(sc.sum_c);
      a.out = kp;
      a.out_ld = h->n_pad;
      a.col_map = cmap;
      a.out_scale = 1.0 / (double)h->m;
      a.err = sc.err;
      tc_grm_kernel<true><<<(unsigned)(h->n_pad / kRows), kThreads, tc_smem_bytes(ng, true), st>>>(
          p->codes_map, a);
      SG_CHECK_LAUNCH();
    }
    h->n_kv += r;
  }
  h->n_kv_launches += 1;
  unsigned int err = 0;
  SG_CUDA(cudaMemcpyAsync(&err, sc.err, sizeof(err), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (err) return fail(SAIGE_TIMEOUT, "tensor-core GRM product: a pipeline wait timed out");
  return Status();
}

}  // namespace saige
