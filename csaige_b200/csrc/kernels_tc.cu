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

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kernels.cuh"
#include "kernels_tc.cuh"

namespace saige {

namespace {

constexpr int kRows = 128;     // MMA M: rows of a CTA tile
constexpr int kKt = 128;       // K per pipeline stage
constexpr int kMaxSA = 4;         // unpacked int8 operand buffers at most
constexpr int kMaxSL = 16;       // load-ring stages at most
constexpr int kUnpackWarps = 8;
constexpr int kThreads = 64 + 32 * kUnpackWarps;  // producer warp, MMA warp, 8 unpack warps
constexpr size_t kSmemBudget = 227 * 1024;
constexpr int kSparseR = 4;    // capacity of the sparse missing-call correction
// Launches with r <= kSparseUseR use it.  Measured on B200 at N=200k, M=150k it is
// slower than the dense indicator product (31 ms vs 13 ms per product at r = 1):
// nearly every word of a warp holds some missing code, so the divergent scan runs
// on almost every word.  It stays selectable here; the dense path is the default.
constexpr int kSparseUseR = 0;
constexpr int kMaxR = 64;      // right-hand sides per launch (3*64 = 192 <= 256 MMA N)
constexpr double kQ = 127.0 * 65536.0;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

struct TcArgs {
  int ng;                   // B tile rows (= MMA N), multiple of 16
  int r;                    // right-hand sides in this launch
  int nk;                   // pipeline stages over K
  int sl;                   // load-ring depth
  int sa;                   // unpacked-ring depth (2 or 4)
  const uint8_t* img_g;     // nk x ng x 128 bytes
  const uint8_t* img_m;     // pass B, dense: c image (same shape)
  const int* img_q;         // sparse: exact int32 q, nk x r x 128
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
  unsigned long long* trace;  // optional pipeline trace of CTA 0 (SAIGE_TC_TRACE=1)
};

constexpr int kTraceStages = 64;
constexpr int kTraceSlots = 8;

// Records %globaltimer for CTA 0, stage k, event slot e when tracing is on.
__device__ __forceinline__ void trace_mark(const TcArgs& a, int k, int e) {
  if (a.trace && blockIdx.x == 0 && k < kTraceStages) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    a.trace[k * kTraceSlots + e] = t;
  }
}

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
template <bool kBackoff>
__device__ __forceinline__ bool mbar_wait_impl(uint32_t bar, uint32_t parity,
                                               volatile int* abort_flag, unsigned int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  uint32_t sleep_ns = 32;
  for (uint32_t polls = 1;; ++polls) {
    if (mbar_try_wait(bar, parity)) return true;
    if (kBackoff) {
      // waiting warps yield their issue slots to the MMA-issuing warp
      __nanosleep(sleep_ns);
      if (sleep_ns < 256) sleep_ns <<= 1;
    }
    if ((polls & 63u) == 0) {  // the clock and the abort flag are checked every 64 polls
      if (*abort_flag) return false;
      if (clock64() - t0 > kWaitCycles) {
        *abort_flag = 1;
        atomicOr(err, 1u);
        return false;
      }
    }
  }
}

// Spin wait for the MMA-issuing thread (on the critical path).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned int* err) {
  return mbar_wait_impl<false>(bar, parity, abort_flag, err);
}

// Wait with exponential back-off (producer, unpack and epilogue warps).
__device__ __forceinline__ bool mbar_wait_sleep(uint32_t bar, uint32_t parity,
                                                volatile int* abort_flag, unsigned int* err) {
  return mbar_wait_impl<true>(bar, parity, abort_flag, err);
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

// Byte-permute selectors of the four 4-sample groups of a device-layout word
// (sample 4j+i at bit 16*(j>>1) + 2*(j&1) + 4i): one nibble per sample.
__device__ __forceinline__ void selectors(uint32_t w, uint32_t& s0, uint32_t& s1, uint32_t& s2,
                                          uint32_t& s3) {
  s0 = w & 0x3333u;
  s1 = (w >> 2) & 0x3333u;
  s2 = (w >> 16) & 0x3333u;
  s3 = (w >> 18) & 0x3333u;
}

// Codes 00,01,10,11 -> genotype bytes {2,0,1,0} and missing bytes {0,1,0,0}.
constexpr uint32_t kLutG = 0x00010002u;
constexpr uint32_t kLutM = 0x00000100u;

// Shared-memory plan (1024-byte aligned):
//   unpacked ring  sa x [A_g 16 KB | A_m 16 KB (dense missing product only)]
//   load ring      sl x [codes 4 KB | B_g ng*128 | B_m ng*128 (pass B, dense) |
//                        Q r*512 (sparse: exact int32 q of the stage's 128 entries)]
//   barriers       FULL[sl] EMPTY_L[sl] UNP[sa] EMPTY_A[sa] ACCF
//   misc           TMEM address, abort flag, sparse missing sums int64 [128][kSparseR]
// The load ring runs up to sl stages ahead of the MMA so that HBM latency is
// covered; two groups of four unpack warps fill alternate unpacked buffers.
//
// Missing calls.  Dense: the missing indicator is a second int8 operand and a
// second MMA (right for many right-hand sides).  Sparse (r <= kSparseR): the
// unpack threads find the ~1% missing codes with bit tricks and add the exact
// int32 q of those entries on CUDA cores, which halves the MMAs and drops the
// indicator tile.
struct SmemPlan {
  uint32_t base, a_stage, l_stage, b_bytes, q_off, bars;
  int sl, sa;
  __device__ uint32_t A_g(int a) const { return base + (uint32_t)a * a_stage; }
  __device__ uint32_t A_m(int a) const { return A_g(a) + kRows * kKt; }
  __device__ uint32_t L(int s) const { return base + (uint32_t)sa * a_stage + (uint32_t)s * l_stage; }
  __device__ uint32_t CODES(int s) const { return L(s); }
  __device__ uint32_t B_g(int s) const { return L(s) + kRows * 32u; }
  __device__ uint32_t B_m(int s) const { return B_g(s) + b_bytes; }
  __device__ uint32_t Q(int s) const { return L(s) + q_off; }
  __device__ uint32_t FULL(int s) const { return bars + 8u * s; }
  __device__ uint32_t EMPTY_L(int s) const { return bars + 8u * (kMaxSL + s); }
  __device__ uint32_t UNP(int a) const { return bars + 8u * (2 * kMaxSL + a); }
  __device__ uint32_t EMPTY_A(int a) const { return bars + 8u * (2 * kMaxSL + kMaxSA + a); }
  __device__ uint32_t ACCF() const { return bars + 8u * (2 * kMaxSL + 2 * kMaxSA); }
  __device__ uint32_t MISC() const { return ACCF() + 8u; }
  __device__ uint32_t MACC() const { return MISC() + 16u; }
};

__host__ __device__ constexpr uint32_t round1k(uint32_t x) { return (x + 1023u) & ~1023u; }

// Offset of the Q tile inside a load stage, and the stage size.
__host__ __device__ constexpr uint32_t plan_q_off(int ng, bool pass_b, bool sparse) {
  return kRows * 32u + (uint32_t)ng * kKt * ((pass_b && !sparse) ? 2u : 1u);
}
__host__ __device__ constexpr uint32_t plan_l_stage(int ng, int r, bool pass_b, bool sparse) {
  return round1k(plan_q_off(ng, pass_b, sparse) + (sparse ? (uint32_t)r * 512u : 0u));
}
__host__ __device__ constexpr uint32_t plan_a_stage(bool sparse) {
  return (sparse ? 1u : 2u) * kRows * kKt;
}

__device__ __forceinline__ int lds_s32(uint32_t addr) {
  int v;
  asm volatile("ld.shared.s32 %0, [%1];" : "=r"(v) : "r"(addr));
  return v;
}

// Fire-and-forget 64-bit add to shared memory.
__device__ __forceinline__ void red_add_u64(uint32_t addr, unsigned long long v) {
  asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}

// Sample index (0..15) of the code at even bit p of a device-layout word.
__device__ __forceinline__ int sample_of_bit(int p) {
  return ((p >> 4) << 3) | (((p >> 1) & 1) << 2) | ((p >> 2) & 3);
}

template <bool kPassB, bool kSparse>
__global__ void __launch_bounds__(kThreads, 1)
    tc_grm_kernel(const __grid_constant__ CUtensorMap codes_map, TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  SmemPlan P;
  P.base = (raw + 1023u) & ~1023u;
  P.b_bytes = (uint32_t)a.ng * kKt;
  P.a_stage = plan_a_stage(kSparse);
  P.q_off = plan_q_off(a.ng, kPassB, kSparse);
  P.l_stage = plan_l_stage(a.ng, a.r, kPassB, kSparse);
  P.sl = a.sl;
  P.sa = a.sa;
  P.bars = P.base + (uint32_t)a.sa * P.a_stage + (uint32_t)a.sl * P.l_stage;
  uint8_t* gen = smem_raw + (P.base - raw);  // generic pointer of P.base
  auto gptr = [&](uint32_t saddr) { return gen + (saddr - P.base); };
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gptr(P.MISC()));
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gptr(P.MISC() + 8u));
  unsigned long long* macc = reinterpret_cast<unsigned long long*>(gptr(P.MACC()));

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const uint32_t acc_cols = (kSparse ? 1u : 2u) * (uint32_t)a.ng;
  uint32_t tmem_cols = 32;
  while (tmem_cols < acc_cols) tmem_cols <<= 1;

  if (kSparse)
    for (int e = threadIdx.x; e < kRows * kSparseR; e += kThreads) macc[e] = 0ull;
  if (threadIdx.x == 0) {
    for (int s = 0; s < a.sl; ++s) {
      mbar_init(P.FULL(s), 1);
      mbar_init(P.EMPTY_L(s), 1);
    }
    for (int s = 0; s < a.sa; ++s) {
      mbar_init(P.UNP(s), kUnpackWarps / 2);  // one arrival per warp of the owning group
      mbar_init(P.EMPTY_A(s), 1);
    }
    mbar_init(P.ACCF(), 1);
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
    // ---------------- producer: codes by TMA, vector tiles by bulk copy ----------------
    if (lane == 0) {
      const uint32_t q_bytes = (uint32_t)a.r * 512u;
      const uint32_t tx = kRows * 32u + P.b_bytes * ((kPassB && !kSparse) ? 2u : 1u) +
                          (kSparse ? q_bytes : 0u);
      int s = 0;
      uint32_t ph = 0;
      for (int k = 0; k < a.nk; ++k) {
        if (k >= a.sl && !mbar_wait_sleep(P.EMPTY_L(s), ph ^ 1u, abort_flag, a.err)) break;
        trace_mark(a, k, 0);  // load issued
        mbar_expect_tx(P.FULL(s), tx);
        // pass A: x = 32-byte column (128 samples) k, y = marker tile;
        // pass B: x = sample tile, y = marker block k.
        const int x = kPassB ? tile * 32 : k * 32;
        const int y = kPassB ? k * kRows : tile * kRows;
        tma_load_2d(P.CODES(s), &codes_map, x, y, P.FULL(s));
        bulk_load(P.B_g(s), a.img_g + (size_t)k * P.b_bytes, P.b_bytes, P.FULL(s));
        if (kPassB && !kSparse)
          bulk_load(P.B_m(s), a.img_m + (size_t)k * P.b_bytes, P.b_bytes, P.FULL(s));
        if (kSparse) bulk_load(P.Q(s), a.img_q + (size_t)k * a.r * 128, q_bytes, P.FULL(s));
        if (++s == a.sl) { s = 0; ph ^= 1u; }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      const uint32_t idesc = i8_idesc(a.ng, kPassB);
      int s = 0, ab = 0;
      uint32_t ph_l = 0, ph_a = 0;  // phase parities of the current load / unpacked slots
      for (int k = 0; k < a.nk; ++k) {
        trace_mark(a, k, 6);  // MMA thread reaches the stage
        if (!mbar_wait(P.UNP(ab), ph_a, abort_flag, a.err)) break;
        if (!mbar_wait(P.FULL(s), ph_l, abort_flag, a.err)) break;
        trace_mark(a, k, 4);  // MMA may issue
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t ag = sw128_desc(P.A_g(ab), kPassB);
        const uint64_t bg = sw128_desc(P.B_g(s), false);
        const uint64_t am = kSparse ? 0ull : sw128_desc(P.A_m(ab), kPassB);
        const uint64_t bm = kSparse ? 0ull : sw128_desc(kPassB ? P.B_m(s) : P.B_g(s), false);
#pragma unroll
        for (int kk = 0; kk < kKt / 32; ++kk) {
          // K advance of 32: 32 bytes along a K-major row, or 32 rows (4 KB) of an MN-major tile
          const uint64_t da = kPassB ? (uint64_t)(kk * 256) : (uint64_t)(kk * 2);
          const uint64_t db = (uint64_t)(kk * 2);
          const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
          mma_i8(tmem_g, ag + da, bg + db, idesc, acc);
          if (!kSparse) mma_i8(tmem_m, am + da, bm + db, idesc, acc);
          if (kk == 0) trace_mark(a, k, 7);  // first MMA issued
        }
        mma_commit(P.EMPTY_A(ab));
        mma_commit(P.EMPTY_L(s));
        trace_mark(a, k, 5);  // MMAs issued
        if (++ab == a.sa) { ab = 0; ph_a ^= 1u; }
        if (++s == a.sl) { s = 0; ph_l ^= 1u; }
      }
      mma_commit(P.ACCF());
    }
  } else {
    // ---------------- unpack (warps 2-9) ----------------
    // group 0 (warps 2-5) takes even stages, group 1 (warps 6-9) odd stages;
    // within a group one thread expands one 32-byte code row (128 entries).
    const int t = threadIdx.x - 64;  // 0..255
    const int grp = t >> 7, row = t & 127;
    const int sw = row & 7;
    long long ms0 = 0, ms1 = 0, ms2 = 0, ms3 = 0;  // pass A sparse: missing sums of this row
    int s = grp % a.sl, ab = grp % a.sa;
    uint32_t ph_l = 0, ph_a = 0;
    for (int k = grp; k < a.nk; k += 2) {
      if (!mbar_wait_sleep(P.FULL(s), ph_l, abort_flag, a.err)) break;
      if (row == 0) trace_mark(a, k, 1);  // codes landed
      if (k >= a.sa && !mbar_wait_sleep(P.EMPTY_A(ab), ph_a ^ 1u, abort_flag, a.err)) break;
      if (row == 0) trace_mark(a, k, 2);  // unpacked buffer free
      const uint4* crow = reinterpret_cast<const uint4*>(gptr(P.CODES(s)) + row * 32);
      const uint4 c0 = crow[0], c1 = crow[1];
      const uint32_t words[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
      uint8_t* ag = gptr(P.A_g(ab)) + row * 128;
      uint8_t* am = kSparse ? nullptr : gptr(P.A_m(ab)) + row * 128;
      const uint32_t qt = P.Q(s);  // shared address of the stage's exact int32 q [r][128]
#pragma unroll
      for (int c = 0; c < 8; ++c) {  // 16-byte chunk c = entries 16c .. 16c+15
        uint32_t s0, s1, s2, s3;
        selectors(words[c], s0, s1, s2, s3);
        uint4 g;
        g.x = __byte_perm(kLutG, 0u, s0);
        g.y = __byte_perm(kLutG, 0u, s1);
        g.z = __byte_perm(kLutG, 0u, s2);
        g.w = __byte_perm(kLutG, 0u, s3);
        const int pos = (c ^ sw) * 16;
        *reinterpret_cast<uint4*>(ag + pos) = g;
        if (!kSparse) {
          uint4 m;
          m.x = __byte_perm(kLutM, 0u, s0);
          m.y = __byte_perm(kLutM, 0u, s1);
          m.z = __byte_perm(kLutM, 0u, s2);
          m.w = __byte_perm(kLutM, 0u, s3);
          *reinterpret_cast<uint4*>(am + pos) = m;
        } else {
          uint32_t mm = words[c] & ~(words[c] >> 1) & 0x55555555u;  // codes 01
          while (mm) {
            const int bit = __ffs(mm) - 1;
            mm &= mm - 1u;
            const int j = c * 16 + sample_of_bit(bit);  // entry of the 128 (always a sample)
            if (!kPassB) {
              // pass A: the row is a marker, j a sample; Q holds q_v of the stage's samples
              const uint32_t qa = qt + 4u * (uint32_t)j;
              ms0 += lds_s32(qa);
              if (a.r > 1) ms1 += lds_s32(qa + 512u);
              if (a.r > 2) ms2 += lds_s32(qa + 1024u);
              if (a.r > 3) ms3 += lds_s32(qa + 1536u);
            } else {
              // pass B: the row is a marker (K); Q holds q_c of the stage's markers
              const uint32_t qa = qt + 4u * (uint32_t)row;
              const uint32_t ma = P.MACC() + 8u * (uint32_t)(j * kSparseR);
#pragma unroll
              for (int r = 0; r < kSparseR; ++r)
                if (r < a.r)
                  red_add_u64(ma + 8u * r, (unsigned long long)(long long)lds_s32(qa + 512u * r));
            }
          }
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(P.UNP(ab));
      if (row == 0) trace_mark(a, k, 3);  // unpack done
      s += 2;
      if (s >= a.sl) { s -= a.sl; ph_l ^= 1u; }
      ab += 2;
      if (ab >= a.sa) { ab -= a.sa; ph_a ^= 1u; }
    }
    if (kSparse) {
      if (!kPassB) {
        const long long ms[kSparseR] = {ms0, ms1, ms2, ms3};
#pragma unroll
        for (int r = 0; r < kSparseR; ++r)
          if (r < a.r) red_add_u64(P.MACC() + 8u * (uint32_t)(row * kSparseR + r), (unsigned long long)ms[r]);
      }
      asm volatile("bar.sync 1, %0;" ::"r"(kUnpackWarps * 32) : "memory");  // unpack warps only
    }
    // ---------------- epilogue: two warps per TMEM lane group ----------------
    __syncwarp();
    const int lg = warp & 3;          // TMEM lane group this warp may access
    const int sub = (warp - 2) >> 2;  // 0 or 1: which half of the column chunks
    const int trow = lg * 32 + lane;
    const bool ok = mbar_wait_sleep(P.ACCF(), 0u, abort_flag, a.err);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t grow = (int64_t)tile * kRows + trow;  // marker (A) or sample (B)
    double rowa = 0.0, rowb = 0.0;
    if (!kPassB) {
      rowa = a.inv_s[grow];
      rowb = a.two_p[grow];
    }
    const uint32_t lane_off = (uint32_t)(lg * 32) << 16;
    for (int r0 = 16 * sub; r0 < a.r; r0 += 32) {
      uint32_t g[48], m[48];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int col = 3 * r0 + 16 * j;
        if (col < a.ng) {
          uint32_t tv[16];
          tmem_ld16(tmem_g + lane_off + (uint32_t)col, tv);
#pragma unroll
          for (int e = 0; e < 16; ++e) g[16 * j + e] = tv[e];
          if (!kSparse) {
            tmem_ld16(tmem_m + lane_off + (uint32_t)col, tv);
#pragma unroll
            for (int e = 0; e < 16; ++e) m[16 * j + e] = tv[e];
          }
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
        const double Mi =
            kSparse ? (double)(long long)macc[trow * kSparseR + (r < kSparseR ? r : 0)]
                    : 65536.0 * (double)(int)m[3 * e] + 256.0 * (double)(int)m[3 * e + 1] +
                          (double)(int)m[3 * e + 2];
        const double S = (double)a.sum_q[r];
        if (!kPassB) {
          // u = (1/s) scale (G - 2p (S - Mi)); explicit roundings (no contraction)
          const double tt = __dsub_rn(G, __dmul_rn(rowb, S - Mi));
          a.out[(int64_t)r * a.out_ld + grow] = __dmul_rn(rowa, __dmul_rn(a.scale_g[r], tt));
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
                   unsigned long long* __restrict__ sum_q, int* __restrict__ qimg) {
  __shared__ long long sh[4];
  const int r = blockIdx.y;
  const int64_t stage = blockIdx.x;
  const int pos = threadIdx.x;
  const int64_t i = stage * 128 + pos;
  const double sc = scale_of(amax[r]);
  const double x = i < len ? v[(int64_t)col_map[r] * ld + i] : 0.0;
  const long long q = __double2ll_rn(x / sc);
  put_limbs(img + stage * (int64_t)ng * 128, r, pos, q);
  if (qimg) qimg[(stage * gridDim.y + r) * 128 + pos] = (int)q;
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
                    uint8_t* __restrict__ img_c, int ng, unsigned long long* __restrict__ sum_c,
                    int* __restrict__ qimg_c) {
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
  if (img_c) put_limbs(img_c + stage * (int64_t)ng * 128, r, pos, qc);
  if (qimg_c) qimg_c[(stage * gridDim.y + r) * 128 + pos] = (int)qc;
  const long long s = block_sum_ll(qc, sh);
  if (threadIdx.x == 0) {
    atomicAdd(&sum_c[r], (unsigned long long)s);
    if (stage == 0) {
      scale_w[r] = sw;
      scale_c[r] = scc;
    }
  }
}

size_t tc_fixed_bytes() {
  return 1024 + 8 * (2 * kMaxSL + 2 * kMaxSA + 1) + 16 + 8 * kRows * kSparseR;
}

// Ring depths for a launch: four unpacked buffers when at least four load
// stages still fit, else two; the load ring takes the rest (at most kMaxSL),
// rounded down to an even depth so that each unpack group owns the same load
// slots at every use and its parity waits never skip a phase.
void tc_rings(int ng, int r, bool pass_b, bool sparse, int& sa, int& sl) {
  const size_t per = plan_l_stage(ng, r, pass_b, sparse);
  const size_t a_stage = plan_a_stage(sparse);
  for (sa = kMaxSA; sa >= 2; sa -= 2) {
    const size_t room = kSmemBudget - tc_fixed_bytes() - (size_t)sa * a_stage;
    sl = (int)std::min<size_t>(kMaxSL, room / per) & ~1;
    if (sl >= 4 || sa == 2) break;
  }
}

size_t tc_smem_bytes(int ng, int r, bool pass_b, bool sparse) {
  int sa, sl;
  tc_rings(ng, r, pass_b, sparse, sa, sl);
  return tc_fixed_bytes() + (size_t)sa * plan_a_stage(sparse) +
         (size_t)sl * plan_l_stage(ng, r, pass_b, sparse);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

}  // namespace

struct TcPlan {
  CUtensorMap codes_map;
  DevBuf img_a, img_w, img_c, img_qa, img_qc, u, scal, cmap, trace;
  bool tracing = false;
};

// Pipeline trace: with SAIGE_TC_TRACE=1 each tensor-core launch records, for
// CTA 0 and its first stages, when loads were issued and landed, when the
// unpacked buffer was free and filled, and when MMAs issued; the per-stage
// offsets (ns from the first load) are printed to stderr.
static Status trace_dump(TcPlan* p, const char* what, cudaStream_t st) {
  std::vector<unsigned long long> t((size_t)kTraceStages * kTraceSlots);
  SG_CUDA(cudaMemcpyAsync(t.data(), p->trace.ptr, t.size() * 8, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  const unsigned long long t0 = t[0];
  fprintf(stderr, "[tc trace] %s: stage load landed free filled may-issue issued reach first-pair (ns)\n", what);
  for (int k = 0; k < kTraceStages; k += (k < 8 ? 1 : 8)) {
    fprintf(stderr, "[tc trace] %3d", k);
    for (int e = 0; e < 8; ++e) {
      const unsigned long long v = t[(size_t)k * kTraceSlots + e];
      fprintf(stderr, " %9lld", v ? (long long)(v - t0) : -1LL);
    }
    fprintf(stderr, "\n");
  }
  SG_CUDA(cudaMemsetAsync(p->trace.ptr, 0, t.size() * 8, st));
  return Status();
}

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
  for (auto kern : {tc_grm_kernel<false, false>, tc_grm_kernel<true, false>,
                    tc_grm_kernel<false, true>, tc_grm_kernel<true, true>}) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSmemBudget);
    if (e != cudaSuccess) {
      delete p;
      return fail(SAIGE_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    }
  }
  const char* tr = getenv("SAIGE_TC_TRACE");
  p->tracing = tr && tr[0] == '1';
  if (p->tracing) {
    Status ts = p->trace.reserve((size_t)kTraceStages * kTraceSlots * 8);
    if (!ts.ok()) {
      delete p;
      return ts;
    }
    SG_CUDA(cudaMemset(p->trace.ptr, 0, (size_t)kTraceStages * kTraceSlots * 8));
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

template <bool kPassB, bool kSparse>
static cudaError_t launch_tc(const TcPlan* p, unsigned grid, const TcArgs& a, cudaStream_t st) {
  tc_grm_kernel<kPassB, kSparse><<<grid, kThreads, tc_smem_bytes(a.ng, a.r, kPassB, kSparse), st>>>(
      p->codes_map, a);
  count_launches(1);
  return cudaGetLastError();
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
  const int rq = std::min(rmax, kSparseR);
  SG_TRY(p->img_a.reserve((size_t)h->n_pad * ng_max));
  SG_TRY(p->img_w.reserve((size_t)h->m_pad * ng_max));
  SG_TRY(p->img_c.reserve((size_t)h->m_pad * ng_max));
  SG_TRY(p->img_qa.reserve((size_t)h->n_pad * rq * sizeof(int)));
  SG_TRY(p->img_qc.reserve((size_t)h->m_pad * rq * sizeof(int)));
  SG_TRY(p->u.reserve((size_t)h->m_pad * rmax * sizeof(double)));
  SG_TRY(p->scal.reserve(9 * kMaxR * 8 + 64));
  SG_TRY(p->cmap.reserve((size_t)q * sizeof(int) + 64));
  Scal sc = carve(p);
  SG_CUDA(cudaMemcpyAsync(p->cmap.ptr, cols.data(), cols.size() * sizeof(int),
                          cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(unsigned int), st));
  // per-pass CUDA-event timing when profiling is on (events on the launching stream)
  std::vector<cudaEvent_t> ev;
  auto mark = [&](cudaEvent_t* e) -> Status {
    if (!h->profiling) return Status();
    SG_CUDA(cudaEventCreate(e));
    ev.push_back(*e);
    SG_CUDA(cudaEventRecord(*e, st));
    return Status();
  };
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_a, ev_b;
  for (size_t c0 = 0; c0 < cols.size(); c0 += kMaxR) {
    const int r = (int)std::min<size_t>(kMaxR, cols.size() - c0);
    const int ng = (int)round_up(3 * r, 16);
    const bool sparse = r <= kSparseUseR;
    const int* cmap = p->cmap.as<int>() + c0;
    SG_CUDA(cudaMemsetAsync(p->scal.ptr, 0, 5 * kMaxR * 8, st));
    SG_CUDA(cudaMemsetAsync(p->img_a.ptr, 0, (size_t)h->n_pad * ng, st));
    // ---- pass A operand ----
    {
      dim3 g1((unsigned)std::min<int64_t>(ceil_div(h->n, 256), 296), (unsigned)r);
      amax_v_kernel<<<g1, 256, 0, st>>>(v, h->n_pad, h->n, cmap, sc.amax_v);
      count_launches(2);
      dim3 g2((unsigned)n_stages_a, (unsigned)r);
      quant_v_kernel<<<g2, 128, 0, st>>>(v, h->n_pad, h->n, cmap, sc.amax_v, sc.scale_v,
                                         p->img_a.as<uint8_t>(), ng, sc.sum_v,
                                         sparse ? p->img_qa.as<int>() : nullptr);
      SG_CHECK_LAUNCH();
    }
    // ---- pass A: u = Z' v ----
    {
      TcArgs a{};
      a.ng = ng;
      a.r = r;
      a.nk = (int)n_stages_a;
      tc_rings(ng, r, false, sparse, a.sa, a.sl);
      a.img_g = p->img_a.as<uint8_t>();
      a.img_q = sparse ? p->img_qa.as<int>() : nullptr;
      a.scale_g = sc.scale_v;
      a.sum_q = reinterpret_cast<const long long*>(sc.sum_v);
      a.two_p = h->two_p;
      a.inv_s = h->inv_s;
      a.out = p->u.as<double>();
      a.out_ld = h->m_pad;
      a.err = sc.err;
      a.trace = p->tracing ? p->trace.as<unsigned long long>() : nullptr;
      const unsigned grid = (unsigned)(h->m_pad / kRows);
      cudaEvent_t t0 = nullptr, t1 = nullptr;
      SG_TRY(mark(&t0));
      const cudaError_t e = sparse ? launch_tc<false, true>(p, grid, a, st)
                                   : launch_tc<false, false>(p, grid, a, st);
      SG_CUDA(e);
      SG_TRY(mark(&t1));
      if (h->profiling) ev_a.emplace_back(t0, t1);
      h->stats.tc_pass_a_launches += 1;
      if (p->tracing) SG_TRY(trace_dump(p, "pass A", st));
    }
    // ---- pass B operands ----
    {
      SG_CUDA(cudaMemsetAsync(p->img_w.ptr, 0, (size_t)h->m_pad * ng, st));
      if (!sparse) SG_CUDA(cudaMemsetAsync(p->img_c.ptr, 0, (size_t)h->m_pad * ng, st));
      dim3 g1((unsigned)std::min<int64_t>(ceil_div(h->m_pad, 256), 296), (unsigned)r);
      count_launches(2);
      amax_wc_kernel<<<g1, 256, 0, st>>>(p->u.as<double>(), h->m_pad, h->m_pad, h->inv_s,
                                         h->two_p, sc.amax_w, sc.amax_c);
      dim3 g2((unsigned)n_stages_b, (unsigned)r);
      quant_wc_kernel<<<g2, 128, 0, st>>>(p->u.as<double>(), h->m_pad, h->inv_s, h->two_p,
                                          sc.amax_w, sc.amax_c, sc.scale_w, sc.scale_c,
                                          p->img_w.as<uint8_t>(),
                                          sparse ? nullptr : p->img_c.as<uint8_t>(), ng, sc.sum_c,
                                          sparse ? p->img_qc.as<int>() : nullptr);
      SG_CHECK_LAUNCH();
    }
    // ---- pass B: y = Z w / M ----
    {
      TcArgs a{};
      a.ng = ng;
      a.r = r;
      a.nk = (int)n_stages_b;
      tc_rings(ng, r, true, sparse, a.sa, a.sl);
      a.img_g = p->img_w.as<uint8_t>();
      a.img_m = sparse ? nullptr : p->img_c.as<uint8_t>();
      a.img_q = sparse ? p->img_qc.as<int>() : nullptr;
      a.scale_g = sc.scale_w;
      a.scale_m = sc.scale_c;
      a.sum_q = reinterpret_cast<const long long*>(sc.sum_c);
      a.out = kp;
      a.out_ld = h->n_pad;
      a.col_map = cmap;
      a.out_scale = 1.0 / (double)h->m;
      a.err = sc.err;
      a.trace = p->tracing ? p->trace.as<unsigned long long>() : nullptr;
      const unsigned grid = (unsigned)(h->n_pad / kRows);
      cudaEvent_t t0 = nullptr, t1 = nullptr;
      SG_TRY(mark(&t0));
      const cudaError_t e = sparse ? launch_tc<true, true>(p, grid, a, st)
                                   : launch_tc<true, false>(p, grid, a, st);
      SG_CUDA(e);
      SG_TRY(mark(&t1));
      if (h->profiling) ev_b.emplace_back(t0, t1);
      h->stats.tc_pass_b_launches += 1;
      if (p->tracing) SG_TRY(trace_dump(p, "pass B", st));
    }
    h->n_kv += r;
  }
  h->n_kv_launches += 1;
  unsigned int err = 0;
  SG_CUDA(cudaMemcpyAsync(&err, sc.err, sizeof(err), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  for (auto& pr : ev_a) {
    float ms = 0.f;
    SG_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
    h->stats.tc_pass_a_ms += ms;
  }
  for (auto& pr : ev_b) {
    float ms = 0.f;
    SG_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
    h->stats.tc_pass_b_ms += ms;
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  if (err) return fail(SAIGE_TIMEOUT, "tensor-core GRM product: a pipeline wait timed out");
  return Status();
}

}  // namespace saige
