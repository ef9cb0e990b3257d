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
// Genotype tiles.  The tensor-core passes read the packed codes as 4 KB tiles
// (128 rows x 128 K entries, 32 bytes per row) stored contiguously in HBM, so
// that each pipeline stage is one sequential 4 KB burst:
//   tiles_m: rows = markers, K = samples  (pass A)
//   tiles_s: rows = samples, K = markers  (pass B, the transpose)
// Both use the device word layout of the row-major copy (entry 4j+i of a
// 16-entry word at bit 16(j>>1) + 2(j&1) + 4i), built once per GRM.
//
// Pipeline (one CTA per 128-row tile, K swept in 128-entry stages):
//   warp 0      bulk-copies the stage's code tile and its vector-limb tile(s)
//               (written beforehand in the 128-byte-swizzled K-major layout)
//               into a shared-memory load ring;
//   warps 2-9   two groups of four warps take alternate stages; each thread
//               expands its row's 128 codes into 128 int8 genotypes and 128
//               int8 missing flags with byte permutes and stores them straight
//               into a TMEM operand slot (tcgen05.st): the A operand never
//               touches shared memory;
//   warp 1      issues tcgen05.mma kind::i8 with A from TMEM and B (limbs)
//               from shared memory, and commits each stage to mbarriers;
//   warps 2-9   finally run the FP64 epilogue from the TMEM accumulators.
// Every mbarrier wait is bounded; a wait that runs out sets an error word the
// host reads back (SAIGE_TIMEOUT).
#include <cuda.h>
#include <math.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <vector>

#include "kernels.cuh"
#include "kernels_tc.cuh"
#include "miss_lists.cuh"
#include "tcgen05.cuh"

namespace saige {

namespace {

using namespace tcx;

constexpr int kRows = 128;                    // MMA M: rows of a CTA tile
constexpr int kKt = 128;                      // K entries per pipeline stage
constexpr uint32_t kTileBytes = kRows * kKt / 4;  // 4 KB of 2-bit codes
constexpr int kMaxSA = 6;                     // TMEM operand slots at most
constexpr int kMaxSL = 24;                    // load-ring stages at most
constexpr int kUnpackWarps = 8;
constexpr int kThreads = 64 + 32 * kUnpackWarps;  // producer warp, MMA warp, 8 unpack warps
constexpr size_t kSmemBudget = 227 * 1024;
constexpr uint32_t kTmemCols = 512;           // the whole TMEM (one CTA per SM)
constexpr uint32_t kSlotCols = 64;            // per slot: 32 columns of genotypes + 32 of flags
constexpr int kMaxR = 64;                     // right-hand sides per launch (3*64 = 192 <= 256 MMA N)
constexpr double kQ = 127.0 * 65536.0;

struct TcArgs {
  int ng;                   // B tile rows (= MMA N), multiple of 16
  int r;                    // right-hand sides in this launch
  int nk;                   // pipeline stages over K
  int sub;                  // 128-entry sub-stages per load stage (1, 2 or 4)
  int sl;                   // load-ring depth in load stages (>= 2)
  int sa;                   // TMEM operand slots, one per sub-stage (a multiple of 2 hb)
  int hb;                   // sub-stages per handoff to the MMA warp (1 or 2)
  int merged;               // 1: one commit per batch (hb == sub == 2, sa == 4, sl >= 3)
  const uint8_t* tiles;     // this pass's code tiles, tile t at (t*tile_ld + k)*4 KB
  int64_t tile_ld;          // tiles from one output tile's row of tiles to the next (>= nk)
  const uint8_t* img_g;     // nk x ng x 128 bytes
  const uint8_t* img_m;     // pass B: c image (same shape)
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
  long long wait_cycles;    // budget of each pipeline wait (0: give up unless already done)
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

// Instruction descriptor: kind::i8, s32 accumulate, signed A and B, both
// K-major, M = 128.
__host__ __device__ constexpr uint32_t i8_idesc(int n) {
  return (2u << 4)                          // c_format = S32
         | (1u << 7)                        // a_format = signed int8
         | (1u << 10)                       // b_format = signed int8
         | ((uint32_t)(n >> 3) << 17)       // N >> 3
         | ((uint32_t)(kRows >> 4) << 24);  // M >> 4
}

// D[tmem] (+)= A[tmem] * B[smem]
__device__ __forceinline__ void mma_i8_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "r"(tmem_a), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Named barriers 1..sa hand operand slot ab from its unpack group (four warps,
// bar.arrive) to the MMA warp (bar.sync).
constexpr int kHandoffThreads = 32 + 32 * (kUnpackWarps / 2);

// 32 consecutive TMEM columns of this thread's lane <- v[0..31].
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, "
      "%29, %30, %31, %32};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]),
      "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]),
      "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]), "r"(v[19]), "r"(v[20]), "r"(v[21]),
      "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]), "r"(v[28]),
      "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}

// Codes 00,01,10,11 -> genotype bytes {2,0,1,0} and missing bytes {0,1,0,0}.
constexpr uint32_t kLutG = 0x00010002u;
constexpr uint32_t kLutM = 0x00000100u;

// Shared-memory plan (1024-byte aligned):
//   load ring  sl x [codes sub x 4 KB | B_g sub x ng*128 | B_m sub x ng*128 (pass B)]
//   barriers   FULL[sl] (load stage landed), LDONE[sl] (its MMAs complete),
//              ADONE[sa] (MMAs reading operand slot complete), ACCF
//   misc       TMEM address, abort flag
// A load stage carries `sub` consecutive 128-entry sub-stages in one
// transaction-counted mbarrier phase: a CTA completes only about one such
// phase per ~550 cycles on sm_100, so 4 KB phases would cap a CTA near
// 15 GB/s; 16 KB and more per phase reach HBM speed.
// TMEM: accumulators G at columns [0, ng), Mi at [ng, 2 ng); operand slots of
// 64 columns (one sub-stage) from column a0 = round_up(2 ng, 32).
struct SmemPlan {
  uint32_t base, l_stage, b_bytes, sub, bars;
  __device__ uint32_t L(int s) const { return base + (uint32_t)s * l_stage; }
  __device__ uint32_t CODES(int s, int t) const { return L(s) + (uint32_t)t * kTileBytes; }
  __device__ uint32_t B_g(int s, int t) const {
    return L(s) + sub * kTileBytes + (uint32_t)t * b_bytes;
  }
  __device__ uint32_t B_m(int s, int t) const {
    return L(s) + sub * (kTileBytes + b_bytes) + (uint32_t)t * b_bytes;
  }
  __device__ uint32_t FULL(int s) const { return bars + 8u * s; }
  __device__ uint32_t LDONE(int s) const { return bars + 8u * (kMaxSL + s); }
  __device__ uint32_t ADONE(int a) const { return bars + 8u * (2 * kMaxSL + a); }
  __device__ uint32_t ACCF() const { return bars + 8u * (2 * kMaxSL + kMaxSA); }
  __device__ uint32_t MISC() const { return ACCF() + 8u; }
};

__host__ __device__ constexpr uint32_t round1k(uint32_t x) { return (x + 1023u) & ~1023u; }

// bytes of one sub-stage in the load ring
__host__ __device__ constexpr uint32_t plan_sub_bytes(int ng, bool pass_b) {
  return kTileBytes + (uint32_t)ng * kKt * (pass_b ? 2u : 1u);
}

__host__ __device__ constexpr uint32_t plan_l_stage(int ng, bool pass_b, int sub) {
  return round1k((uint32_t)sub * plan_sub_bytes(ng, pass_b));
}

__host__ __device__ constexpr uint32_t tmem_a0(int ng) { return ((uint32_t)(2 * ng) + 31u) & ~31u; }

// Expands one 16-entry code word into 16 genotype bytes (g[0..3]) and 16
// missing-flag bytes (m[0..3]), entries in order.  PRMT reads only the low
// 16 bits of its selector, so each selector is one nibble group.
__device__ __forceinline__ void expand_word(uint32_t w, uint32_t* g, uint32_t* m) {
  const uint32_t lo = w & 0x33333333u;         // entries 0-3 (bits 0-15), 8-11 (bits 16-31)
  const uint32_t hi = (w >> 2) & 0x33333333u;  // entries 4-7, 12-15
  const uint32_t lo2 = lo >> 16, hi2 = hi >> 16;
  g[0] = __byte_perm(kLutG, 0u, lo);
  g[1] = __byte_perm(kLutG, 0u, hi);
  g[2] = __byte_perm(kLutG, 0u, lo2);
  g[3] = __byte_perm(kLutG, 0u, hi2);
  m[0] = __byte_perm(kLutM, 0u, lo);
  m[1] = __byte_perm(kLutM, 0u, hi);
  m[2] = __byte_perm(kLutM, 0u, lo2);
  m[3] = __byte_perm(kLutM, 0u, hi2);
}

// kHb: sub-stages per handoff (a.hb), a template parameter so that the batch loops
// unroll to straight-line code.  kMerged (with kHb == 2 and two sub-stages per load
// stage): one commit per batch, on the load stage's LDONE barrier, frees both the load
// slot and the batch's two operand slots.  A tcgen05.commit leaves the tensor pipe idle
// for ~200 cycles (measured: 8 MMAs of M=128, N=128, K=32 per sub-stage took ~830
// cycles with 1.5 commits per sub-stage and no handoff at all, 32 MMAs ~2,300), so the
// merged batches — 16 MMAs per commit instead of 8 per 1.5 — keep it busier.
template <bool kPassB, int kHb, bool kMerged>
__global__ void __launch_bounds__(kThreads, 1) tc_grm_kernel(TcArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  SmemPlan P;
  P.base = (raw + 1023u) & ~1023u;
  P.b_bytes = (uint32_t)a.ng * kKt;
  P.sub = (uint32_t)a.sub;
  P.l_stage = plan_l_stage(a.ng, kPassB, a.sub);
  P.bars = P.base + (uint32_t)a.sl * P.l_stage;
  uint8_t* gen = smem_raw + (P.base - raw);  // generic pointer of P.base
  auto gptr = [&](uint32_t saddr) { return gen + (saddr - P.base); };
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gptr(P.MISC()));
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gptr(P.MISC() + 8u));

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < a.sl; ++s) {
      mbar_init(P.FULL(s), 1);
      mbar_init(P.LDONE(s), 1);
    }
    for (int s = 0; s < a.sa; ++s) mbar_init(P.ADONE(s), 1);
    mbar_init(P.ACCF(), 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t tmem_g = tmem, tmem_m = tmem + (uint32_t)a.ng;
  const uint32_t tmem_a = tmem + tmem_a0(a.ng);

  if (warp == 0) {
    // ---------------- producer: code tiles and limb tiles by bulk copy ----------------
    if (lane == 0) {
      const int n_load = (a.nk + a.sub - 1) / a.sub;
      const uint8_t* codes = a.tiles + (size_t)tile * a.tile_ld * kTileBytes;
      int S = 0;
      uint32_t ph = 0;  // (J / sl) & 1
      int issued = 0;   // load stages whose copies were issued
      for (int J = 0; J < n_load; ++J) {
        // the slot is free once the MMAs of load stage J - sl completed
        if (J >= a.sl && !mbar_wait_sleep(P.LDONE(S), ph ^ 1u, abort_flag, a.err, a.wait_cycles))
          break;
        if (J < kTraceStages) trace_mark(a, J, 0);  // load issued
        const int k0 = J * a.sub;
        const uint32_t cnt = (uint32_t)min(a.sub, a.nk - k0);
        mbar_expect_tx(P.FULL(S), cnt * (kTileBytes + P.b_bytes * (kPassB ? 2u : 1u)));
        bulk_load(P.CODES(S, 0), codes + (size_t)k0 * kTileBytes, cnt * kTileBytes, P.FULL(S));
        for (uint32_t t = 0; t < cnt; ++t) {  // limb tiles: one copy per sub-stage (<= 24 KB)
          bulk_load(P.B_g(S, t), a.img_g + (size_t)(k0 + t) * P.b_bytes, P.b_bytes, P.FULL(S));
          if (kPassB)
            bulk_load(P.B_m(S, t), a.img_m + (size_t)(k0 + t) * P.b_bytes, P.b_bytes, P.FULL(S));
        }
        issued = J + 1;
        if (++S == a.sl) { S = 0; ph ^= 1u; }
      }
      // Before the CTA exits, every issued copy has landed: load stage J completes
      // phase (J / sl) & 1 of FULL(J % sl), and only the last sl issued stages can
      // still be in flight (stage J was issued after stage J - sl was consumed).  On
      // the normal path these phases completed long ago and the waits return at once.
      for (int J = issued > a.sl ? issued - a.sl : 0; J < issued; ++J)
        mbar_wait_drain(P.FULL(J % a.sl), (uint32_t)((J / a.sl) & 1), a.err);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    // The whole warp takes each filled operand slot from its unpack group through
    // a named barrier and lane 0 issues the stage's MMAs.  The issuing thread
    // performs no memory access while its MMAs are in flight: on sm_100 such an
    // access waits for all of them to complete, which would drain the tensor
    // pipe at every stage.  One commit per stage releases both the load slot
    // and the operand slot.
    // Ring positions advance incrementally: no division in the loop.
    const uint32_t idesc = i8_idesc(a.ng);
    int t = 0, s = 0, ab = 0;  // sub-stage within the load stage, load slot, operand slot
    // (lane 0) the last load stage and sub-stage whose LDONE / ADONE was committed
    int j_done = -1, k_done = -1;
    // One named-barrier handoff per batch of hb sub-stages (slots ab .. ab + hb - 1,
    // barrier 1 + ab / hb): the warp waits once, then lane 0 issues the whole batch.
    for (int k = 0; k < a.nk;) {
      if (lane == 1) {
        trace_mark(a, k, 6);  // MMA warp reaches the stage
        if (a.trace && blockIdx.x == 0 && k < kTraceStages)
          a.trace[k * kTraceSlots + 7] = (unsigned long long)clock64();  // SM clock at the same point
      }
      named_bar_sync(1 + (ab >> (kHb - 1)), kHandoffThreads);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (lane == 1) trace_mark(a, k, 4);  // MMA may issue
      // After an abort no further MMA is issued (the handoffs still run, in step with
      // the unpack groups).  Lane 1 reads the flag: lane 0, which has MMAs in flight,
      // makes no memory access.
      const int aborted = __shfl_sync(0xffffffffu, lane == 1 ? *abort_flag : 0, 1);
      const int k_batch = k;
#pragma unroll
      for (int j = 0; j < kHb; ++j, ++k) {
        if (kHb > 1 && k >= a.nk) break;
        if (lane == 0 && !aborted) {
          // genotype and missing-flag MMAs alternate (two independent accumulators
          // pipeline; grouping each accumulator's MMAs measured 15-40 % slower), and
          // each sub-stage is committed as soon as its MMAs are issued, so that its
          // operand and load slots free up one sub-stage earlier than a batch commit
          const uint64_t bg = sw128_desc(P.B_g(s, t));
          const uint64_t bm = kPassB ? sw128_desc(P.B_m(s, t)) : bg;
          const uint32_t ag = tmem_a + (uint32_t)ab * kSlotCols, am = ag + 32u;
#pragma unroll
          for (int kk = 0; kk < kKt / 32; ++kk) {
            // K advance of 32 int8: 8 TMEM columns of A, 32 bytes (2 x 16 B) along a B row
            const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
            mma_i8_ts(tmem_g, ag + 8u * kk, bg + 2u * kk, idesc, acc);
            mma_i8_ts(tmem_m, am + 8u * kk, bm + 2u * kk, idesc, acc);
          }
          if (!kMerged) {
            mma_commit(P.ADONE(ab));
            k_done = k;
          }
          if (t == a.sub - 1 || k == a.nk - 1) {
            mma_commit(P.LDONE(s));
            j_done = k / a.sub;
          }
        }
        if (++t == a.sub) {
          t = 0;
          if (++s == a.sl) s = 0;
        }
        if (++ab == a.sa) ab = 0;
      }
      __syncwarp();
      if (lane == 1) trace_mark(a, k_batch, 5);  // MMAs issued
    }
    if (lane == 0) {
      mma_commit(P.ACCF());
      // A commit's mbarrier arrival is performed when its MMAs complete, in no set order
      // with the other commits: the epilogue's wait on ACCF does not cover the last
      // LDONE / ADONE arrivals, and one still in flight when the CTA exits would land in
      // the shared memory of the next CTA on this SM.  So wait for the last committed
      // phase of every such barrier (bounded) before the CTA can finish.
      for (int ls = 0; ls < a.sl; ++ls) {
        if (j_done < ls) continue;  // slot never committed
        const int j = j_done - (j_done - ls) % a.sl;
        mbar_wait_drain(P.LDONE(ls), (uint32_t)((j / a.sl) & 1), a.err);
      }
      if (!kMerged)
        for (int as = 0; as < a.sa; ++as) {
          if (k_done < as) continue;
          const int kk2 = k_done - (k_done - as) % a.sa;
          mbar_wait_drain(P.ADONE(as), (uint32_t)((kk2 / a.sa) & 1), a.err);
        }
    }
  } else {
    // ---------------- unpack (warps 2-9) ----------------
    // group 0 (warps 2-5) takes even stages, group 1 (warps 6-9) odd stages;
    // a warp may only address its own TMEM lane group (warp % 4), so thread
    // `lane` of warp w expands row 32 (w % 4) + lane.
    const int grp = (warp - 2) >> 2;
    const int lg = warp & 3;
    const int row = lg * 32 + lane;
    const uint32_t lane_off = (uint32_t)(lg * 32) << 16;
    bool live = true;  // false once a wait gave up: the remaining stages only hand over
    // Group g takes the batches b = g, g + 2, ... of hb sub-stages (sub-stages b hb ..
    // b hb + hb - 1).  Ring positions of the current sub-stage advance one sub-stage at
    // a time (no division in the loop).
    constexpr int hb = kHb;
    int t = 0, s = 0, ab = 0;
    uint32_t ph_l = 0;  // phase parity of FULL(s) for the current sub-stage
    uint32_t ph_a = 0;  // (k / sa) & 1
    auto step = [&]() {
      if (++t == a.sub) {
        t = 0;
        if (++s == a.sl) { s = 0; ph_l ^= 1u; }
      }
      if (++ab == a.sa) { ab = 0; ph_a ^= 1u; }
    };
    for (int j = 0; j < grp * hb; ++j) step();
    for (int kb = grp * hb; kb < a.nk; kb += 2 * hb) {
      const int bar = 1 + (ab >> (hb - 1));  // the batch's named barrier
#pragma unroll
      for (int j = 0; j < hb; ++j) {
        const int k = kb + j;
        if (hb == 1 || k < a.nk) {
          // Operand slot ab is free once the MMAs of its previous use (sub-stage k - sa)
          // completed; merged: both slots of the batch once the MMAs of the batch two
          // before (this group's previous batch, load stage kb/2 - 2, in the slot two
          // back) completed.  This wait comes before the one on the codes: a group sees
          // only every other phase of a load slot that the two groups share (an odd ring
          // depth), so FULL(s) may still be a phase behind — its previous load in flight
          // — and its parity would then already read as this load's.  Once the MMA warp
          // has taken sub-stage k - sa (merged: batch kb/2 - 2), every load stage up to
          // it was seen complete, which covers load stage k/sub - sl for every accepted
          // ring shape ((sl - 1) sub + 1 >= sa; merged: sl >= 3), so the parity below is
          // unambiguous.  The LDONE phase is the latest of its slot, since the next use
          // of the slot, load stage kb/2 - 2 + sl, follows this batch.
          if (!kMerged) {
            if (live && k >= a.sa)
              live = mbar_wait_sleep(P.ADONE(ab), ph_a ^ 1u, abort_flag, a.err, a.wait_cycles);
          } else if (j == 0 && live && kb >= 2 * hb) {
            const int s2 = s >= 2 ? s - 2 : s - 2 + a.sl;
            const uint32_t ph2 = s >= 2 ? ph_l : (ph_l ^ 1u);
            live = mbar_wait_sleep(P.LDONE(s2), ph2, abort_flag, a.err, a.wait_cycles);
          }
          if (live) live = mbar_wait_sleep(P.FULL(s), ph_l, abort_flag, a.err, a.wait_cycles);
          if (live && row == 0) trace_mark(a, k, 1);  // codes landed
          live = __all_sync(0xffffffffu, live);  // warp-uniform: the barrier calls below must agree
          if (live) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (row == 0) trace_mark(a, k, 2);  // operand slot free
            const uint32_t crow = P.CODES(s, t) + (uint32_t)row * 32u;
            const uint4 c0 = lds128(crow), c1 = lds128(crow + 16u);
            const uint32_t words[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
            uint32_t g[32], m[32];
#pragma unroll
            for (int c = 0; c < 8; ++c) expand_word(words[c], g + 4 * c, m + 4 * c);
            const uint32_t slot = tmem_a + lane_off + (uint32_t)ab * kSlotCols;
            tmem_st32(slot, g);
            tmem_st32(slot + 32u, m);
            tmem_wait_st();
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            if (row == 0) trace_mark(a, k, 3);  // unpack done
          }
        }
        step();
      }
      // Every batch is handed over, also after an abort, so that the MMA warp never
      // waits for an arrival that does not come.  While live, the wait on the slots'
      // previous use keeps this group at most one use ahead of the MMA warp on its
      // named barrier; after an abort bar.sync does that instead.
      if (live)
        named_bar_arrive(bar, kHandoffThreads);
      else
        named_bar_sync(bar, kHandoffThreads);
#pragma unroll
      for (int j = 0; j < hb; ++j) step();  // the other group's batch
    }
    // ---------------- epilogue: two warps per TMEM lane group ----------------
    __syncwarp();
    const int sub = grp;  // 0 or 1: which half of the column chunks
    const int trow = row;
    // The MMA warp always commits ACCF after its last MMA (none after an abort), so
    // this wait also ensures that no MMA is in flight when the TMEM is freed.
    const bool ok = mbar_wait_drain(P.ACCF(), 0u, a.err) && !*abort_flag;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int64_t grow = (int64_t)tile * kRows + trow;  // marker (A) or sample (B)
    double rowa = 0.0, rowb = 0.0;
    if (!kPassB) {
      rowa = a.inv_s[grow];
      rowb = a.two_p[grow];
    }
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
          tmem_ld16(tmem_m + lane_off + (uint32_t)col, tv);
#pragma unroll
          for (int e = 0; e < 16; ++e) m[16 * j + e] = tv[e];
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
                 "r"(kTmemCols));
  }
}

// ---------------------------------------------------------------------------
// genotype tiles
// ---------------------------------------------------------------------------
// Bit offset of entry e (0..15) of a 16-entry word in the device word layout.
__device__ __forceinline__ int entry_bit(int e) {
  const int j = e >> 2, i = e & 3;
  return 16 * (j >> 1) + 2 * (j & 1) + 4 * i;
}

// tiles_m[(mt * n_kt + kt)] row r = row-major row mt*128 + r, words kt*8 .. kt*8+7,
// for the marker tiles mt0 + blockIdx.y.
__global__ void __launch_bounds__(256)
    pack_tiles_kernel(const uint32_t* __restrict__ geno, int64_t wpr, int64_t n_kt, int64_t mt0,
                      uint8_t* __restrict__ tiles) {
  const int64_t kt = blockIdx.x, mt = mt0 + blockIdx.y;
  const int r = threadIdx.x >> 1, half = threadIdx.x & 1;
  const uint4 v = *reinterpret_cast<const uint4*>(geno + (mt * kRows + r) * wpr + kt * 8 + half * 4);
  *reinterpret_cast<uint4*>(tiles + (mt * n_kt + kt) * kTileBytes + r * 32 + half * 16) = v;
}

// tiles_s[(st * s_ld + mt)] row r = sample st*128 + r, word j = markers
// mt*128 + 16j .. +15, read from tiles_m[(mt * n_st + st)], for the marker tiles
// mt0 + blockIdx.x.
__global__ void __launch_bounds__(256)
    transpose_tiles_kernel(const uint8_t* __restrict__ tiles_m, int64_t n_st, int64_t s_ld,
                           int64_t mt0, uint8_t* __restrict__ tiles_s) {
  __shared__ __align__(16) uint32_t src[kTileBytes / 4];
  __shared__ __align__(16) uint32_t dst[kTileBytes / 4];
  const int64_t mt = mt0 + blockIdx.x, st = blockIdx.y;
  const uint4* s4 = reinterpret_cast<const uint4*>(tiles_m + (mt * n_st + st) * kTileBytes);
  reinterpret_cast<uint4*>(src)[threadIdx.x] = s4[threadIdx.x];
  __syncthreads();
  // output word (r, j): thread handles r = idx & 127, j = idx >> 7 for idx = t, t+256, ...
  for (int idx = threadIdx.x; idx < kRows * 8; idx += 256) {
    const int r = idx & 127, j = idx >> 7;
    const int sb = entry_bit(r & 15);
    uint32_t w = 0;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const uint32_t sw = src[(16 * j + e) * 8 + (r >> 4)];  // marker row 16j+e, sample word r/16
      w |= ((sw >> sb) & 3u) << entry_bit(e);
    }
    dst[r * 8 + j] = w;
  }
  __syncthreads();
  reinterpret_cast<uint4*>(tiles_s + (st * s_ld + mt) * kTileBytes)[threadIdx.x] =
      reinterpret_cast<const uint4*>(dst)[threadIdx.x];
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

// Limb rows 3r, 3r+1, 3r+2 of a stage image (K-major, 128-byte swizzle).
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

// One block = one 128-entry stage of one column: quantise v, write the limbs
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

// ---------------------------------------------------------------------------
// Single-column products on the CUDA cores.  With one column the tensor-core
// passes are bound by their fixed per-stage cost (eight MMAs and the unpack of a
// 4 KB code tile for three limb columns), so one column costs nearly what 42 do.
// These kernels form the same exact integer sums with dp4a — the limbs of q as
// int8 planes, genotypes and missing flags expanded four at a time by byte
// permutes — and apply the same FP64 epilogue, so their results are bit-identical
// to the tensor-core path's.  With the missing-call lists of the handle
// (miss_lists.cuh) the flag sums give way to int64 sums over the ~1 % missing calls,
// a third fewer instructions per entry for the same integers.
// ---------------------------------------------------------------------------
// prmt tables of the NEGATED genotype (codes 00, 01, 10, 11 -> -2, 0, -1, 0) and of
// the missing flag (01 -> 1).  A selector nibble holds the code either in its bits
// 0-1 (value c: byte c of x) or in its bits 2-3 (value 4c: byte 0 or byte 4 (y),
// sign-replicated when the code's high bit is set — 10 gives sign(x.byte0), 11
// sign(y.byte0)); both tables give the right byte in both positions, so the
// selectors need masks but no shifts.
constexpr uint32_t kNegGenoX = 0x00FF00FEu, kNegGenoY = 0u;
constexpr uint32_t kMissX = 0x00000100u, kMissY = 0x00000001u;
constexpr int kSrWarpMarkers = 8;                        // pass A: markers per warp
constexpr int kSrBlockMarkers = 8 * kSrWarpMarkers;      // pass A: markers per block
constexpr int kSrWords = 1024;                           // pass A: sample words staged per round
constexpr int kSrChunk = 2048;  // markers of limb planes staged per pass-B round
// error word bit of a one-column product: a missing-call list entry out of range (the
// entry is skipped; timeouts of the tensor-core pipeline set other bits)
constexpr unsigned int kSrListErr = 1u << 30;
// Missing-call entries of a pass-A segment staged at once in shared memory (a block's 64
// markers x 16,384 samples: ~10,500 calls at 1 % missing); larger segments take several
// pieces.  (Pass B reads its segments, ~5,200 calls per chunk, from global memory: staging
// them cost it more resident blocks than the uncoalesced reads cost; 3.89 against 3.09 ms
// per pass at 200,000 x 150,000.)
constexpr int kPieceA = 12288;
// dynamic shared memory of sr_pass_a_kernel: three planes of kSrWords 16-byte words, and
// with the missing-call lists a piece of entries and one int64 counter per marker
constexpr size_t sr_pass_a_smem(bool lists) {
  return 3 * kSrWords * 16 + (lists ? kPieceA * 4 + kSrBlockMarkers * 8 : 0);
}
static_assert(kSamplePad % 256 == 0, "pass B of one column takes sample tiles in pairs");

__device__ __forceinline__ uint32_t prmt(uint32_t x, uint32_t y, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(x), "r"(y), "r"(sel));
  return d;
}

// The four 4-entry groups of a packed word (device layout: entry 4j+i at bit
// 16(j>>1) + 2(j&1) + 4i; group g = entries 4g..4g+3) as four bytes each of -g and
// of the missing flag.
__device__ __forceinline__ void sr_expand(uint32_t w, int neg_g[4], int miss[4]) {
  const uint32_t hi = w >> 16;
  const uint32_t sel[4] = {w & 0x3333u, w & 0xCCCCu, hi & 0x3333u, hi & 0xCCCCu};
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    neg_g[g] = (int)prmt(kNegGenoX, kNegGenoY, sel[g]);
    miss[g] = (int)prmt(kMissX, kMissY, sel[g]);
  }
}

// Asynchronous 4-byte copies global -> shared (cp.async), their commit, and the wait
// for all of this thread's committed copies.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Entries [p0, p0 + n) of a list copied into buf (shared memory) by the block's nt
// threads, asynchronously: complete after cp_async_wait_all and a barrier.
__device__ __forceinline__ void stage_piece(uint32_t* buf, const uint32_t* __restrict__ ent,
                                            int64_t p0, int n, int t, int nt) {
  for (int i = t; i < n; i += nt) cp_async4(buf + i, ent + p0 + i);
  cp_async_commit();
}

// One thread's share of a segment of missing-call entries (tag << bits | position),
// ascending: the contiguous slice [e0 + t L, e0 + (t + 1) L) of [e0, e1) with L =
// ceil((e1 - e0) / nt).  Consecutive entries mostly share a tag (a row or a sample), so
// the thread sums value(position) per run of equal tags in int64 and adds each run to
// counters[tag] with one shared-memory atomic.  An entry whose tag or position is out of
// range (tag >= n_tags, position >= n_pos) sets kSrListErr in err and is skipped.
template <class Value>
__device__ __forceinline__ void add_slice(const uint32_t* ent, int64_t e0, int64_t e1,
                                          int t, int nt, int bits, uint32_t n_tags, uint32_t n_pos,
                                          unsigned long long* counters, unsigned int* err,
                                          Value value) {
  const int64_t len = (e1 - e0 + nt - 1) / nt;
  const int64_t lo = e0 + (int64_t)t * len;
  const int64_t hi = lo + len < e1 ? lo + len : e1;
  const uint32_t pmask = (1u << bits) - 1u;
  uint32_t tag = 0xFFFFFFFFu;
  long long acc = 0;
#pragma unroll 4
  for (int64_t e = lo; e < hi; ++e) {
    const uint32_t x = ent[e];
    const uint32_t g = x >> bits, pos = x & pmask;
    if (g >= n_tags || pos >= n_pos) {
      atomicOr(err, kSrListErr);
      continue;
    }
    if (g != tag) {
      if (tag != 0xFFFFFFFFu) atomicAdd(&counters[tag], (unsigned long long)acc);
      tag = g;
      acc = 0;
    }
    acc += value(pos);
  }
  if (tag != 0xFFFFFFFFu) atomicAdd(&counters[tag], (unsigned long long)acc);
}

// The same groups as bytes of -g only (the missing sums come from the lists).
__device__ __forceinline__ void sr_expand_g(uint32_t w, int neg_g[4]) {
  const uint32_t hi = w >> 16;
  const uint32_t sel[4] = {w & 0x3333u, w & 0xCCCCu, hi & 0x3333u, hi & 0xCCCCu};
#pragma unroll
  for (int g = 0; g < 4; ++g) neg_g[g] = (int)prmt(kNegGenoX, kNegGenoY, sel[g]);
}

// q = rint(x / scale) as in quant_v_kernel, into three int8 planes (l2, l1, l0) of
// length n_pad (zero past len), and sum q.
__global__ void __launch_bounds__(256)
    sr_quant_v_kernel(const double* __restrict__ v, int64_t len, int64_t n_pad,
                      const unsigned long long* __restrict__ amax, double* __restrict__ scale_out,
                      int8_t* __restrict__ planes, unsigned long long* __restrict__ sum_q) {
  __shared__ long long sh[8];
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  const double sc = scale_of(amax[0]);
  long long q = 0;
  if (i < n_pad) {
    const double x = i < len ? v[i] : 0.0;
    q = __double2ll_rn(x / sc);
    int l2, l1, l0;
    limbs(q, l2, l1, l0);
    planes[i] = (int8_t)l2;
    planes[n_pad + i] = (int8_t)l1;
    planes[2 * n_pad + i] = (int8_t)l0;
  }
  long long t = q;
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int k = 0; k < 8; ++k) s += sh[k];
    atomicAdd(sum_q, (unsigned long long)s);
    if (blockIdx.x == 0) scale_out[0] = sc;
  }
}

// w = u inv_s, c = w 2p quantised as in quant_wc_kernel into planes (w: l2 l1 l0,
// c: l2 l1 l0; length m_pad each) and, when qc32 is given, qc as int32 (|qc| <= 127 *
// 2^16); and sum qc.
__global__ void __launch_bounds__(256)
    sr_quant_wc_kernel(const double* __restrict__ u, int64_t m_pad,
                       const double* __restrict__ inv_s, const double* __restrict__ two_p,
                       const unsigned long long* __restrict__ amax_w,
                       const unsigned long long* __restrict__ amax_c, double* __restrict__ scale_w,
                       double* __restrict__ scale_c, int8_t* __restrict__ planes,
                       int32_t* __restrict__ qc32, unsigned long long* __restrict__ sum_c) {
  __shared__ long long sh[8];
  const int64_t m = (int64_t)blockIdx.x * 256 + threadIdx.x;
  const double sw = scale_of(amax_w[0]), scc = scale_of(amax_c[0]);
  long long qc = 0;
  if (m < m_pad) {
    const double w = u[m] * inv_s[m];
    const double c = w * two_p[m];
    const long long qw = __double2ll_rn(w / sw);
    qc = __double2ll_rn(c / scc);
    int l2, l1, l0;
    limbs(qw, l2, l1, l0);
    planes[m] = (int8_t)l2;
    planes[m_pad + m] = (int8_t)l1;
    planes[2 * m_pad + m] = (int8_t)l0;
    limbs(qc, l2, l1, l0);
    planes[3 * m_pad + m] = (int8_t)l2;
    planes[4 * m_pad + m] = (int8_t)l1;
    planes[5 * m_pad + m] = (int8_t)l0;
    if (qc32) qc32[m] = (int32_t)qc;
  }
  long long t = qc;
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int k = 0; k < 8; ++k) s += sh[k];
    atomicAdd(sum_c, (unsigned long long)s);
    if (blockIdx.x == 0) {
      scale_w[0] = sw;
      scale_c[0] = scc;
    }
  }
}

// Pass A of one column: block = 64 markers x all samples, warp = 8 markers.  The
// limb planes of q are staged in shared memory kSrWords words (16 samples each) at a
// time and shared by the block's warps; each lane keeps the six sums of its warp's 8
// markers over its words, and the warp's sums are finished as in the tensor-core
// epilogue.  With kLists the lanes keep the three genotype sums only: after each chunk
// the block adds q (rebuilt from its staged limbs) over the missing calls of its markers
// in the chunk — one segment of miss_ent, each entry (marker in block) << bits | (sample
// in chunk) — into per-marker int64 counters: the same integer Mi the flag sums give.
template <bool kLists>
__global__ void __launch_bounds__(256, 2)
    sr_pass_a_kernel(const uint32_t* __restrict__ geno, int64_t wpr,
                     const int8_t* __restrict__ planes, int64_t n_pad,
                     const unsigned long long* __restrict__ sum_q,
                     const double* __restrict__ scale_v, const double* __restrict__ two_p,
                     const double* __restrict__ inv_s, const uint32_t* __restrict__ miss_ent,
                     const int64_t* __restrict__ miss_seg, int64_t nch, int bits,
                     unsigned int* __restrict__ err, double* __restrict__ u) {
  constexpr int kSums = kLists ? 3 : 6;
  // dynamic shared memory (sr_pass_a_smem bytes): the three staged limb planes, then
  // with kLists the per-marker missing sums and a piece of the chunk's entries
  extern __shared__ uint4 sr_dyn[];
  uint4(*sp)[kSrWords] = reinterpret_cast<uint4(*)[kSrWords]>(sr_dyn);
  unsigned long long* mi_s = reinterpret_cast<unsigned long long*>(sr_dyn + 3 * kSrWords);
  uint32_t* piece = reinterpret_cast<uint32_t*>(mi_s + kSrBlockMarkers);
  if constexpr (kLists) {
    if (threadIdx.x < kSrBlockMarkers) mi_s[threadIdx.x] = 0ull;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t m0 = (int64_t)blockIdx.x * kSrBlockMarkers + warp * kSrWarpMarkers;
  const uint32_t* rows = geno + m0 * wpr;
  int acc[kSrWarpMarkers][kSums];
#pragma unroll
  for (int k = 0; k < kSrWarpMarkers; ++k)
#pragma unroll
    for (int j = 0; j < kSums; ++j) acc[k][j] = 0;
  const int64_t n_words = n_pad / 16;
  for (int64_t c0 = 0; c0 < n_words; c0 += kSrWords) {
    const int cn = n_words - c0 < kSrWords ? (int)(n_words - c0) : kSrWords;
    int64_t e0 = 0, e1 = 0;  // kLists: this chunk's segment
    if constexpr (kLists) {
      const int64_t* sg = miss_seg + (int64_t)blockIdx.x * nch + c0 / kSrWords;
      e0 = sg[0];
      e1 = sg[1];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 3 * kSrWords; t += 256) {
      const int pl = t / kSrWords, k = t % kSrWords;
      sp[pl][k] = k < cn ? __ldg(reinterpret_cast<const uint4*>(planes + pl * n_pad) + c0 + k)
                         : make_uint4(0u, 0u, 0u, 0u);
    }
    // kLists: the segment's first piece lands while the dense loop runs
    if constexpr (kLists)
      stage_piece(piece, miss_ent, e0, (int)(e1 - e0 < kPieceA ? e1 - e0 : kPieceA), threadIdx.x,
                  256);
    __syncthreads();
#pragma unroll 4
    for (int t = lane; t < cn; t += 32) {
      uint32_t w[kSrWarpMarkers];
#pragma unroll
      for (int k = 0; k < kSrWarpMarkers; ++k) w[k] = __ldg(rows + k * wpr + c0 + t);
      const uint4 a2 = sp[0][t], a1 = sp[1][t], a0 = sp[2][t];
      const int l2[4] = {(int)a2.x, (int)a2.y, (int)a2.z, (int)a2.w};
      const int l1[4] = {(int)a1.x, (int)a1.y, (int)a1.z, (int)a1.w};
      const int l0[4] = {(int)a0.x, (int)a0.y, (int)a0.z, (int)a0.w};
#pragma unroll
      for (int k = 0; k < kSrWarpMarkers; ++k) {
        if constexpr (kLists) {
          int gbs[4];
          sr_expand_g(w[k], gbs);
#pragma unroll
          for (int g = 0; g < 4; ++g) {
            acc[k][0] = __dp4a(gbs[g], l2[g], acc[k][0]);
            acc[k][1] = __dp4a(gbs[g], l1[g], acc[k][1]);
            acc[k][2] = __dp4a(gbs[g], l0[g], acc[k][2]);
          }
        } else {
          int gbs[4], mbs[4];
          sr_expand(w[k], gbs, mbs);
#pragma unroll
          for (int g = 0; g < 4; ++g) {
            const int gb = gbs[g], mb = mbs[g];
            acc[k][0] = __dp4a(gb, l2[g], acc[k][0]);
            acc[k][1] = __dp4a(gb, l1[g], acc[k][1]);
            acc[k][2] = __dp4a(gb, l0[g], acc[k][2]);
            acc[k][3] = __dp4a(mb, l2[g], acc[k][3]);
            acc[k][4] = __dp4a(mb, l1[g], acc[k][4]);
            acc[k][5] = __dp4a(mb, l0[g], acc[k][5]);
          }
        }
      }
    }
    if constexpr (kLists) {
      const int8_t* p2 = reinterpret_cast<const int8_t*>(sp[0]);
      const int8_t* p1 = reinterpret_cast<const int8_t*>(sp[1]);
      const int8_t* p0 = reinterpret_cast<const int8_t*>(sp[2]);
      for (int64_t q0 = e0; q0 < e1; q0 += kPieceA) {  // uniform over the block
        const int n = (int)(e1 - q0 < kPieceA ? e1 - q0 : kPieceA);
        if (q0 != e0) {  // a later piece: after the last one's slices are done
          __syncthreads();
          stage_piece(piece, miss_ent, q0, n, threadIdx.x, 256);
        }
        cp_async_wait_all();
        __syncthreads();
        add_slice(piece, 0, n, threadIdx.x, 256, bits, kSrBlockMarkers, 16u * (uint32_t)cn, mi_s,
                  err, [&](uint32_t s) {
                    return 65536LL * p2[s] + 256LL * p1[s] + (long long)p0[s];
                  });
      }
    }
  }
  if constexpr (kLists) __syncthreads();
#pragma unroll
  for (int k = 0; k < kSrWarpMarkers; ++k)
#pragma unroll
    for (int j = 0; j < kSums; ++j)
      for (int o = 16; o > 0; o >>= 1) acc[k][j] += __shfl_xor_sync(0xffffffffu, acc[k][j], o);
  const double S = (double)(long long)sum_q[0];
#pragma unroll
  for (int k = 0; k < kSrWarpMarkers; ++k) {
    if (lane != k) continue;
    const int64_t m = m0 + k;
    // the genotype sums were formed with -g; Mi is the same integer either way
    const double G = -(65536.0 * (double)acc[k][0] + 256.0 * (double)acc[k][1] + (double)acc[k][2]);
    double Mi;
    if constexpr (kLists)
      Mi = (double)(long long)mi_s[warp * kSrWarpMarkers + k];
    else
      Mi = 65536.0 * (double)acc[k][kSums - 3] + 256.0 * (double)acc[k][kSums - 2] +
           (double)acc[k][kSums - 1];
    const double tt = __dsub_rn(G, __dmul_rn(two_p[m], S - Mi));
    u[m] = __dmul_rn(inv_s[m], __dmul_rn(scale_v[0], tt));
  }
}

// Pass B of one column: block = two 128-sample tiles of tiles_s, thread = one sample of
// each (the limb words it loads serve both).  The marker limb planes are staged in
// shared memory kSrChunk markers at a time.  With kLists the c planes give way to qc
// itself (qc32), and after each chunk the block adds qc over the missing calls of its
// 256 samples in the chunk — one segment of miss_ent, each entry (sample in block) <<
// bits | (marker in chunk) — into per-sample int64 counters: the integer Mi the flag
// sums give.
template <bool kLists>
__global__ void __launch_bounds__(128)
    sr_pass_b_kernel(const uint8_t* __restrict__ tiles_s, int64_t n_mt, int64_t s_ld,
                     const int8_t* __restrict__ planes, int64_t m_pad,
                     const unsigned long long* __restrict__ sum_c,
                     const double* __restrict__ scale_w, const double* __restrict__ scale_c,
                     const int32_t* __restrict__ qc32, const uint32_t* __restrict__ miss_ent,
                     const int64_t* __restrict__ miss_seg, int64_t nch, int bits,
                     unsigned int* __restrict__ err, double out_scale, double* __restrict__ out) {
  constexpr int kPlanes = kLists ? 3 : 6;
  __shared__ __align__(16) int8_t sp[kPlanes][kSrChunk];
  __shared__ __align__(16) int32_t sq[kLists ? kSrChunk : 4];
  const int64_t st0 = 2 * (int64_t)blockIdx.x;
  const int r = threadIdx.x;
  int acc[2][kPlanes];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int e = 0; e < kPlanes; ++e) acc[h][e] = 0;
  __shared__ unsigned long long mi_s[kLists ? 2 * kRows : 1];
  if constexpr (kLists) {
    mi_s[r] = 0ull;
    mi_s[kRows + r] = 0ull;
  }
  for (int64_t mt0 = 0; mt0 < n_mt; mt0 += kSrChunk / 128) {
    const int64_t base = mt0 * 128;
    const int64_t len = m_pad - base < kSrChunk ? m_pad - base : (int64_t)kSrChunk;
    int64_t e0 = 0, e1 = 0;  // kLists: this chunk's segment
    if constexpr (kLists) {
      const int64_t* sg = miss_seg + (int64_t)blockIdx.x * nch + mt0 / (kSrChunk / 128);
      e0 = sg[0];
      e1 = sg[1];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < kPlanes * (kSrChunk / 16); t += 128) {
      const int pl = t / (kSrChunk / 16), k = t % (kSrChunk / 16);
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (16 * k < len)
        v = __ldg(reinterpret_cast<const uint4*>(planes + (int64_t)pl * m_pad + base) + k);
      reinterpret_cast<uint4*>(sp[pl])[k] = v;
    }
    if constexpr (kLists) {
      for (int t = threadIdx.x; t < kSrChunk / 4; t += 128) {
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (4 * t < len) v = __ldg(reinterpret_cast<const uint4*>(qc32 + base) + t);
        reinterpret_cast<uint4*>(sq)[t] = v;
      }
    }
    __syncthreads();
    const int64_t mt_end = mt0 + kSrChunk / 128 < n_mt ? mt0 + kSrChunk / 128 : n_mt;
#pragma unroll 2
    for (int64_t mt = mt0; mt < mt_end; ++mt) {
      uint32_t words[2][8];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint4* row = reinterpret_cast<const uint4*>(
            tiles_s + ((st0 + h) * s_ld + mt) * kTileBytes + (int64_t)r * 32);
        const uint4 h0 = __ldg(row), h1 = __ldg(row + 1);
        words[h][0] = h0.x; words[h][1] = h0.y; words[h][2] = h0.z; words[h][3] = h0.w;
        words[h][4] = h1.x; words[h][5] = h1.y; words[h][6] = h1.z; words[h][7] = h1.w;
      }
      const int off = (int)(mt - mt0) * 128;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int mk = off + 16 * j;
        const uint4 w2 = *reinterpret_cast<const uint4*>(sp[0] + mk);
        const uint4 w1 = *reinterpret_cast<const uint4*>(sp[1] + mk);
        const uint4 w0 = *reinterpret_cast<const uint4*>(sp[2] + mk);
        const int W2[4] = {(int)w2.x, (int)w2.y, (int)w2.z, (int)w2.w};
        const int W1[4] = {(int)w1.x, (int)w1.y, (int)w1.z, (int)w1.w};
        const int W0[4] = {(int)w0.x, (int)w0.y, (int)w0.z, (int)w0.w};
        if constexpr (kLists) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            int gbs[4];
            sr_expand_g(words[h][j], gbs);
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              acc[h][0] = __dp4a(gbs[g], W2[g], acc[h][0]);
              acc[h][1] = __dp4a(gbs[g], W1[g], acc[h][1]);
              acc[h][2] = __dp4a(gbs[g], W0[g], acc[h][2]);
            }
          }
        } else {
          const uint4 c2 = *reinterpret_cast<const uint4*>(sp[kPlanes - 3] + mk);
          const uint4 c1 = *reinterpret_cast<const uint4*>(sp[kPlanes - 2] + mk);
          const uint4 c0 = *reinterpret_cast<const uint4*>(sp[kPlanes - 1] + mk);
          const int C2[4] = {(int)c2.x, (int)c2.y, (int)c2.z, (int)c2.w};
          const int C1[4] = {(int)c1.x, (int)c1.y, (int)c1.z, (int)c1.w};
          const int C0[4] = {(int)c0.x, (int)c0.y, (int)c0.z, (int)c0.w};
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            int gbs[4], mbs[4];
            sr_expand(words[h][j], gbs, mbs);
#pragma unroll
            for (int g = 0; g < 4; ++g) {
              acc[h][0] = __dp4a(gbs[g], W2[g], acc[h][0]);
              acc[h][1] = __dp4a(gbs[g], W1[g], acc[h][1]);
              acc[h][2] = __dp4a(gbs[g], W0[g], acc[h][2]);
              acc[h][kPlanes - 3] = __dp4a(mbs[g], C2[g], acc[h][kPlanes - 3]);
              acc[h][kPlanes - 2] = __dp4a(mbs[g], C1[g], acc[h][kPlanes - 2]);
              acc[h][kPlanes - 1] = __dp4a(mbs[g], C0[g], acc[h][kPlanes - 1]);
            }
          }
        }
      }
    }
    if constexpr (kLists) {
      add_slice(miss_ent, e0, e1, threadIdx.x, 128, bits, 2u * kRows, (uint32_t)len, mi_s, err,
                [&](uint32_t mk) { return (long long)sq[mk]; });
    }
  }
  if constexpr (kLists) __syncthreads();
  const double S = (double)(long long)sum_c[0];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    // the genotype sums were formed with -g; Mi is the same integer either way
    const double G =
        -(65536.0 * (double)acc[h][0] + 256.0 * (double)acc[h][1] + (double)acc[h][2]);
    double Mi;
    if constexpr (kLists)
      Mi = (double)(long long)mi_s[h * kRows + r];
    else
      Mi = 65536.0 * (double)acc[h][kPlanes - 3] + 256.0 * (double)acc[h][kPlanes - 2] +
           (double)acc[h][kPlanes - 1];
    out[(st0 + h) * 128 + r] = __dmul_rn(
        out_scale, __dsub_rn(__dmul_rn(scale_w[0], G), __dmul_rn(scale_c[0], S - Mi)));
  }
}

size_t tc_fixed_bytes() { return 1024 + 8 * (2 * kMaxSL + kMaxSA + 1) + 16; }

struct Rings {
  int sub, sl, sa, hb;
  bool merged = false;  // one commit per batch of two sub-stages (kMerged)
};

// Ring shapes for a launch: load stages of up to four sub-stages (16 KB of
// codes) while at least two such stages fit in shared memory; as many load
// stages as fit (at most kMaxSL); as many TMEM operand slots as the
// accumulators leave room for (at most kMaxSA, even, so that each unpack group
// owns its slots and named barriers).
// Operand slots (even) that a ring of sl load stages of sub sub-stages accepts: at
// most (sl - 1) sub + 1, so that the slot-reuse wait of an unpack group implies its
// load slot's previous load landed.
int slots_for_ring(int slots, int sl, int sub) {
  return std::min(slots, (sl - 1) * sub + 1) & ~1;
}

Rings tc_rings(int ng, bool pass_b) {
  Rings g;
  const size_t room = kSmemBudget - tc_fixed_bytes();
  // batches of two sub-stages with one commit each (the load stage = the batch), where
  // four operand slots and a ring of three such stages fit
  const int slots = std::min<int>(kMaxSA, (int)((kTmemCols - tmem_a0(ng)) / kSlotCols));
  if (slots >= 4 && room / plan_l_stage(ng, pass_b, 2) >= 3) {
    g.sub = 2;
    g.sl = (int)std::min<size_t>(kMaxSL, room / plan_l_stage(ng, pass_b, 2));
    g.sa = 4;
    g.hb = 2;
    g.merged = true;
    return g;
  }
  // the most sub-stages per load stage that still leave a ring of four load stages:
  // at the bench size the autotuner's trials put the shapes with a 2-3 stage ring
  // 2-25 % behind (pass B at 43-64 columns most), and no deeper ring of fewer
  // sub-stages lost more than 1 %
  g.sub = 4;
  while (g.sub > 1 && room / plan_l_stage(ng, pass_b, g.sub) < 4) g.sub >>= 1;
  g.sl = (int)std::min<size_t>(kMaxSL, room / plan_l_stage(ng, pass_b, g.sub));
  g.sa = slots_for_ring(std::min<int>(kMaxSA, (int)((kTmemCols - tmem_a0(ng)) / kSlotCols)),
                        g.sl, g.sub);
  // one sub-stage per handoff (two, a tuner candidate, measured 1-5 % slower)
  g.hb = 1;
  return g;
}

}  // namespace

struct TcPlan {
  DevBuf tiles_m, tiles_s, img_a, img_w, img_c, u, scal, cmap, trace;
  int64_t s_ld = 0;  // tiles_s: marker tiles per sample tile (>= m_pad / 128)
  bool tracing = false;
  // one-column products: the missing-call lists and qc as int32 (m_pad) for pass B's
  // sums over them
  MissLists miss;
  DevBuf sr_qc;
};

// The missing-call lists cost about two products' time to build (four passes over the
// codes) and 8 bytes per missing call, while a fit runs four or five one-column products:
// a handle builds them at the first one-column product of its second AI-REML fit, so a
// single fit (with its variance ratio) keeps the dense flag sums and repeated fits on a
// handle (refits, LOCO) take the lists.
// SAIGE_SR_LISTS: 0 keeps the dense missing-flag sums, 2 builds the lists at a handle's
// first one-column product, otherwise (default) in its second fit.
static int sr_lists_mode() {
  const char* e = getenv("SAIGE_SR_LISTS");
  if (!e || !e[0]) return 1;
  return e[0] == '0' ? 0 : (e[0] == '2' ? 2 : 1);
}

// Pipeline trace: with SAIGE_TC_TRACE=1 each tensor-core launch records, for
// CTA 0 and its first stages, when loads were issued and landed, when the
// operand slot was free and filled, and when MMAs issued; the per-stage
// offsets (ns from the first load) are printed to stderr.
static Status trace_dump(TcPlan* p, const char* what, cudaStream_t st) {
  std::vector<unsigned long long> t((size_t)kTraceStages * kTraceSlots);
  SG_CUDA(cudaMemcpyAsync(t.data(), p->trace.ptr, t.size() * 8, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  const unsigned long long t0 = t[0];
  fprintf(stderr, "[tc trace] %s: stage load landed free filled may-issue issued reach (ns) | SM clock (MHz)\n", what);
  for (int k = 0; k < kTraceStages; k += (k < 8 ? 1 : 8)) {
    fprintf(stderr, "[tc trace] %3d", k);
    for (int e = 0; e < 7; ++e) {
      const unsigned long long v = t[(size_t)k * kTraceSlots + e];
      fprintf(stderr, " %9lld", v ? (long long)(v - t0) : -1LL);
    }
    // effective SM clock between the MMA warp's arrivals at stage 0 and stage k
    const unsigned long long c0 = t[7], ck = t[(size_t)k * kTraceSlots + 7];
    const unsigned long long g0 = t[6], gk = t[(size_t)k * kTraceSlots + 6];
    fprintf(stderr, " | %6.0f", (k > 0 && gk > g0) ? (double)(ck - c0) * 1e3 / (double)(gk - g0) : 0.0);
    fprintf(stderr, "\n");
  }
  SG_CUDA(cudaMemsetAsync(p->trace.ptr, 0, t.size() * 8, st));
  return Status();
}

// Builds the two tile copies of the packed genotypes (marker-major for pass A,
// sample-major for pass B) from the row-major copy, on the handle's stream.
// Tiles of the marker tiles [mt0, mt1) from the row-major rows, on stream st.
static Status tiles_range(saige_grm* h, TcPlan* p, int64_t mt0, int64_t mt1, cudaStream_t st) {
  if (mt1 <= mt0) return Status();
  const int64_t n_st = h->n_pad / kKt;
  pack_tiles_kernel<<<dim3((unsigned)n_st, (unsigned)(mt1 - mt0)), 256, 0, st>>>(
      h->geno, h->wpr, n_st, mt0, p->tiles_m.as<uint8_t>());
  SG_CHECK_LAUNCH();
  transpose_tiles_kernel<<<dim3((unsigned)(mt1 - mt0), (unsigned)n_st), 256, 0, st>>>(
      p->tiles_m.as<uint8_t>(), n_st, p->s_ld, mt0, p->tiles_s.as<uint8_t>());
  SG_CHECK_LAUNCH();
  count_launches(2);
  return Status();
}

static Status reserve_tiles(saige_grm* h, TcPlan* p, int64_t n_mt) {
  const size_t bytes = (size_t)n_mt * (size_t)(h->n_pad / kKt) * kTileBytes;
  SG_TRY(p->tiles_m.reserve(bytes));
  SG_TRY(p->tiles_s.reserve(bytes));
  p->s_ld = n_mt;
  return Status();
}

// A new plan with the kernels' attributes set and, when asked for, the trace buffer;
// the tiles are the caller's.
static Status tc_plan_new(TcPlan** out) {
  TcPlan* p = new TcPlan();
  auto bail = [&](Status s) {
    delete p;
    return s;
  };
  for (auto kern : {tc_grm_kernel<false, 1, false>, tc_grm_kernel<true, 1, false>,
                    tc_grm_kernel<false, 2, false>, tc_grm_kernel<true, 2, false>,
                    tc_grm_kernel<false, 2, true>, tc_grm_kernel<true, 2, true>}) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kSmemBudget);
    if (e != cudaSuccess)
      return bail(fail(SAIGE_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e)));
  }
  for (bool lists : {false, true}) {
    cudaError_t e = cudaFuncSetAttribute(
        lists ? sr_pass_a_kernel<true> : sr_pass_a_kernel<false>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sr_pass_a_smem(lists));
    if (e != cudaSuccess)
      return bail(fail(SAIGE_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e)));
  }
  const char* tr = getenv("SAIGE_TC_TRACE");
  p->tracing = tr && tr[0] == '1';
  if (p->tracing) {
    Status ts = p->trace.reserve((size_t)kTraceStages * kTraceSlots * 8);
    if (!ts.ok()) return bail(ts);
    // (tracing only) cleared on the legacy stream and waited for, since the handle's
    // non-blocking stream would not order itself after it
    cudaError_t e = cudaMemset(p->trace.ptr, 0, (size_t)kTraceStages * kTraceSlots * 8);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return bail(fail(SAIGE_ECUDA, "cudaMemset: %s", cudaGetErrorString(e)));
  }
  *out = p;
  return Status();
}

static Status tc_init(saige_grm* h) {
  if (h->tc) return Status();
  TcPlan* p = nullptr;
  SG_TRY(tc_plan_new(&p));
  PhaseTimer tm;
  Status bs = reserve_tiles(h, p, h->m_pad / kRows);
  if (bs.ok()) bs = tiles_range(h, p, 0, h->m_pad / kRows, h->stream);
  if (!bs.ok()) {
    delete p;
    return bs;
  }
  tm.mark(" tc tiles");
  h->tc = p;
  return Status();
}

Status tc_stream_begin(saige_grm* h, int64_t rows_cap) {
  if (h->tc) return fail(SAIGE_EINVAL, "tensor-core tiles already built");
  TcPlan* p = nullptr;
  SG_TRY(tc_plan_new(&p));
  Status s = reserve_tiles(h, p, ceil_div(rows_cap, (int64_t)kRows));
  if (!s.ok()) {
    delete p;
    return s;
  }
  h->tc = p;
  return Status();
}

Status tc_stream_tiles(saige_grm* h, int64_t mt0, int64_t mt1, cudaStream_t st) {
  if (!h->tc || mt1 > h->tc->s_ld) return fail(SAIGE_EINVAL, "tile range beyond the reserved tiles");
  return tiles_range(h, h->tc, mt0, mt1, st);
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

// Budget of each pipeline wait in SM cycles; saige_tc_set_wait_budget changes it.
std::atomic<long long> g_tc_wait_cycles{kWaitCycles};

template <bool kPassB>
static cudaError_t launch_tc(unsigned grid, const TcArgs& args, cudaStream_t st) {
  TcArgs a = args;
  a.wait_cycles = g_tc_wait_cycles.load(std::memory_order_relaxed);
  if (a.hb < 1 || a.hb > 2 || a.sa < 2 * a.hb || a.sa % (2 * a.hb) || a.sa > kMaxSA ||
      a.sl < 2 || a.sl > kMaxSL || a.sub < 1 ||
      a.sub > 4)
    return cudaErrorInvalidValue;
  if (a.merged && !(a.hb == 2 && a.sub == 2 && a.sa == 4 && a.sl >= 3))
    return cudaErrorInvalidValue;
  // an unpack group may wait on a load slot's codes only once the slot's previous load
  // is known to have landed (see the unpack loop): (sl - 1) sub + 1 >= sa
  if (!a.merged && (a.sl - 1) * a.sub + 1 < a.sa) return cudaErrorInvalidValue;
  const size_t smem = tc_fixed_bytes() + (size_t)a.sl * plan_l_stage(a.ng, kPassB, a.sub);
  if (smem > kSmemBudget) return cudaErrorInvalidValue;
  if (a.merged)
    tc_grm_kernel<kPassB, 2, true><<<grid, kThreads, smem, st>>>(a);
  else if (a.hb == 2)
    tc_grm_kernel<kPassB, 2, false><<<grid, kThreads, smem, st>>>(a);
  else
    tc_grm_kernel<kPassB, 1, false><<<grid, kThreads, smem, st>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

// ---- ring-shape autotuner ----------------------------------------------------
// The ring shape (sub-stages per load stage, load-ring depth, TMEM operand slots)
// does not change a product's result — the sums are exact integers and the epilogue
// is per element — only its speed.  So the tuning needs no launches of its own: the
// first launches of each key — pass, ng and the launch's size class (log2 of its 4 KB
// stages) — in the process each run the real product with the next candidate shape
// (sub 4, 2, 1 with the deepest ring the shared memory holds; one or two sub-stages per
// handoff where four operand slots fit; tc_rings' choice first), timed with CUDA events
// that are read at the key's next launch; once every candidate has run, the fastest is
// kept for the later launches.  Launches of fewer than kTuneMinStages stages keep the
// fixed choice of tc_rings, as does SAIGE_TC_AUTOTUNE=0 (=2 tunes every size).
// SAIGE_TIMING=1 logs each timed candidate.
namespace {

struct TuneKey {
  int dev, pass_b, ng, size_class;
  bool operator<(const TuneKey& o) const {
    if (dev != o.dev) return dev < o.dev;
    if (pass_b != o.pass_b) return pass_b < o.pass_b;
    if (ng != o.ng) return ng < o.ng;
    return size_class < o.size_class;
  }
};

constexpr double kTuneMinStages = 1 << 20;  // ~4 GB of code tiles per launch

int size_class(double stages) {
  int c = 0;
  while (stages >= 2.0) {
    stages *= 0.5;
    ++c;
  }
  return c;
}

struct TuneState {
  std::vector<Rings> cand;
  std::vector<float> ms;               // per candidate; < 0: not timed (launch refused)
  size_t next = 0;                     // next candidate to run
  int pending = -1;                    // candidate whose events wait to be read
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool done = false;
  Rings best{};
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneState> g_tune;
std::atomic<int64_t> g_tune_trials{0};

// SAIGE_TC_AUTOTUNE: 0 off, 2 every launch size, otherwise (default) launches of at
// least kTuneMinStages stages.
int autotune_level() {
  const char* e = getenv("SAIGE_TC_AUTOTUNE");
  if (!e || !e[0]) return 1;
  return e[0] == '0' ? 0 : (e[0] == '2' ? 2 : 1);
}

std::vector<Rings> tc_candidates(int ng, bool pass_b) {
  std::vector<Rings> out;
  const size_t room = kSmemBudget - tc_fixed_bytes();
  const Rings base = tc_rings(ng, pass_b);
  out.push_back(base);  // the fixed choice first
  const int slots = std::min<int>(kMaxSA, (int)((kTmemCols - tmem_a0(ng)) / kSlotCols)) & ~1;
  for (int sub : {4, 2, 1}) {
    const size_t ls = plan_l_stage(ng, pass_b, sub);
    if (2 * ls > room) continue;
    Rings g;
    g.sub = sub;
    g.sl = (int)std::min<size_t>(kMaxSL, room / ls);
    g.sa = slots_for_ring(slots, g.sl, sub);
    g.hb = 1;
    if (g.sa < 2) continue;
    out.push_back(g);
    if (g.sa >= 4) {  // the same ring with two sub-stages per handoff (four slots)
      g.hb = 2;
      g.sa = 4;
      out.push_back(g);
      if (sub == 2 && g.sl >= 3) {  // and one commit per batch
        g.merged = true;
        out.push_back(g);
      }
    }
  }
  // the fixed choice appears once
  for (size_t i = 1; i < out.size();) {
    const Rings& g = out[i];
    if (g.sub == base.sub && g.sl == base.sl && g.sa == base.sa && g.hb == base.hb &&
        g.merged == base.merged)
      out.erase(out.begin() + (std::ptrdiff_t)i);
    else
      ++i;
  }
  return out;
}

}  // namespace

// Launches pass kPassB with the tuned ring shape of its key, tuning it first when the
// key is new.  a carries everything but the ring shape.
template <bool kPassB>
static Status launch_tc_tuned(int dev, unsigned grid, TcArgs a, cudaStream_t st) {
  const Rings fixed = tc_rings(a.ng, kPassB);
  const double stages = (double)grid * (double)a.nk;
  const int level = autotune_level();
  if (level == 0 || (level == 1 && stages < kTuneMinStages)) {
    a.sub = fixed.sub;
    a.sl = fixed.sl;
    a.sa = fixed.sa;
    a.hb = fixed.hb;
    a.merged = fixed.merged ? 1 : 0;
    SG_CUDA(launch_tc<kPassB>(grid, a, st));
    return Status();
  }
  const TuneKey key{dev, kPassB ? 1 : 0, a.ng, size_class(stages)};
  auto use = [&](const Rings& g) {
    a.sub = g.sub;
    a.sl = g.sl;
    a.sa = g.sa;
    a.hb = g.hb;
    a.merged = g.merged ? 1 : 0;
  };
  // the state is held under the lock through the (asynchronous) launch, so that one
  // key's candidates and events are used by one launch at a time
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneState& ts = g_tune[key];
  if (ts.done) {
    use(ts.best);
    SG_CUDA(launch_tc<kPassB>(grid, a, st));
    return Status();
  }
  if (ts.cand.empty()) {
    ts.cand = tc_candidates(a.ng, kPassB);
    ts.ms.assign(ts.cand.size(), -1.f);
    SG_CUDA(cudaEventCreate(&ts.e0));
    SG_CUDA(cudaEventCreate(&ts.e1));
  }
  const char* tlog = getenv("SAIGE_TIMING");
  const bool log = tlog && tlog[0] == '1';
  if (ts.pending >= 0) {  // the previous candidate's launch of this key has long been queued
    SG_CUDA(cudaEventSynchronize(ts.e1));
    float ms = 0.f;
    SG_CUDA(cudaEventElapsedTime(&ms, ts.e0, ts.e1));
    ts.ms[(size_t)ts.pending] = ms;
    const Rings& g = ts.cand[(size_t)ts.pending];
    if (log)
      fprintf(stderr, "[saige tune] pass %c ng %d grid %u nk %d: sub %d sl %d hb %d merged %d -> %.3f ms\n",
              kPassB ? 'B' : 'A', a.ng, grid, a.nk, g.sub, g.sl, g.hb, g.merged ? 1 : 0, ms);
    ts.pending = -1;
  }
  while (ts.next < ts.cand.size()) {
    const size_t c = ts.next++;
    use(ts.cand[c]);
    SG_CUDA(cudaEventRecord(ts.e0, st));
    const cudaError_t le = launch_tc<kPassB>(grid, a, st);
    if (le != cudaSuccess) {  // a shape the launch refuses: next candidate
      (void)cudaGetLastError();
      continue;
    }
    SG_CUDA(cudaEventRecord(ts.e1, st));
    ts.pending = (int)c;
    g_tune_trials += 1;
    return Status();
  }
  // every candidate has run: keep the fastest
  int bi = -1;
  for (size_t c = 0; c < ts.cand.size(); ++c)
    if (ts.ms[c] >= 0.f && (bi < 0 || ts.ms[c] < ts.ms[(size_t)bi])) bi = (int)c;
  ts.best = bi >= 0 ? ts.cand[(size_t)bi] : fixed;
  ts.done = true;
  use(ts.best);
  SG_CUDA(launch_tc<kPassB>(grid, a, st));
  return Status();
}

int64_t tc_autotune_trials() { return g_tune_trials.load(); }

int64_t tc_missing_listed(const saige_grm* h) {
  return h->tc && h->tc->miss.state == 1 ? h->tc->miss.total : -1;
}

void tc_set_wait_budget(long long cycles) {
  g_tc_wait_cycles.store(cycles < 0 ? kWaitCycles : cycles, std::memory_order_relaxed);
}

Status tc_product(saige_grm* h, const double* v, double* kp, int q, const int32_t* active,
                  cudaStream_t st) {
  SG_TRY(tc_init(h));
  TcPlan* p = h->tc;
  std::vector<int> cols;
  for (int c = 0; c < q; ++c)
    if (!active || active[c] == kColActive) cols.push_back(c);
  if (cols.empty()) return Status();
  if (st != h->stream) {
    // the tiles were built on the handle's stream
    cudaEvent_t built;
    SG_CUDA(cudaEventCreateWithFlags(&built, cudaEventDisableTiming));
    SG_CUDA(cudaEventRecord(built, h->stream));
    SG_CUDA(cudaStreamWaitEvent(st, built, 0));
    cudaEventDestroy(built);
  }
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
  // per-pass CUDA-event timing when profiling is on (events on the launching stream)
  std::vector<cudaEvent_t> ev;
  auto mark = [&](cudaEvent_t* e) -> Status {
    if (!h->profiling) return Status();
    SG_CUDA(cudaEventCreate(e));
    ev.push_back(*e);
    SG_CUDA(cudaEventRecord(*e, st));
    return Status();
  };
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_a, ev_b, ev_s;
  const char* sc_env = getenv("SAIGE_SC");
  const bool single = cols.size() == 1 && !(sc_env && sc_env[0] == '0');
  if (single) {
    // one column: both passes on the CUDA cores (same integer sums, same epilogue)
    int8_t* planes_a = p->img_a.as<int8_t>();  // 3 x n_pad limb planes of q
    int8_t* planes_b = p->img_w.as<int8_t>();  // 6 x m_pad limb planes of qw, qc
    double* u = p->u.as<double>();
    const int lmode = sr_lists_mode();
    if (p->miss.state == 0 && (lmode == 2 || (lmode == 1 && h->n_fits >= 2)))
      SG_TRY(miss_lists_build(h, p->tiles_s.as<uint8_t>(), p->s_ld,
                              MissShape{kSrBlockMarkers, kSrWords, 2 * kRows, kSrChunk}, &p->miss,
                              st));
    const bool lists = p->miss.state == 1 && lmode != 0;
    int32_t* qc32 = nullptr;
    if (lists) {
      SG_TRY(p->sr_qc.reserve((size_t)h->m_pad * sizeof(int32_t)));
      qc32 = p->sr_qc.as<int32_t>();
    }
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    SG_TRY(mark(&t0));
    SG_CUDA(cudaMemsetAsync(p->scal.ptr, 0, 5 * kMaxR * 8, st));
    const dim3 g1a((unsigned)std::min<int64_t>(ceil_div(h->n, 256), 296), 1u);
    amax_v_kernel<<<g1a, 256, 0, st>>>(v, h->n_pad, h->n, p->cmap.as<int>(), sc.amax_v);
    sr_quant_v_kernel<<<(unsigned)ceil_div(h->n_pad, 256), 256, 0, st>>>(
        v + (int64_t)cols[0] * h->n_pad, h->n, h->n_pad, sc.amax_v, sc.scale_v, planes_a, sc.sum_v);
    if (lists)
      sr_pass_a_kernel<true><<<(unsigned)(h->m_pad / kSrBlockMarkers), 256, sr_pass_a_smem(true),
                               st>>>(
          h->geno, h->wpr, planes_a, h->n_pad, sc.sum_v, sc.scale_v, h->two_p, h->inv_s,
          p->miss.a_ent.as<uint32_t>(), p->miss.a_seg.as<int64_t>(), p->miss.a_nch, p->miss.a_bits,
          sc.err, u);
    else
      sr_pass_a_kernel<false><<<(unsigned)(h->m_pad / kSrBlockMarkers), 256, sr_pass_a_smem(false),
                                st>>>(
          h->geno, h->wpr, planes_a, h->n_pad, sc.sum_v, sc.scale_v, h->two_p, h->inv_s, nullptr,
          nullptr, 0, 0, nullptr, u);
    SG_CHECK_LAUNCH();
    if (h->masked) SG_CUDA(mask_rows_f64(u, h->m_pad, 1, h->excl.as<uint8_t>(), h->m, st));
    const dim3 g1b((unsigned)std::min<int64_t>(ceil_div(h->m_pad, 256), 296), 1u);
    amax_wc_kernel<<<g1b, 256, 0, st>>>(u, h->m_pad, h->m_pad, h->inv_s, h->two_p, sc.amax_w,
                                        sc.amax_c);
    sr_quant_wc_kernel<<<(unsigned)ceil_div(h->m_pad, 256), 256, 0, st>>>(
        u, h->m_pad, h->inv_s, h->two_p, sc.amax_w, sc.amax_c, sc.scale_w, sc.scale_c, planes_b,
        qc32, sc.sum_c);
    // two sample tiles per block (n_pad is a multiple of 512: an even tile count)
    const unsigned grid_b = (unsigned)(h->n_pad / (2 * kRows));
    const double out_scale = 1.0 / (double)(h->masked ? h->m_active : h->m_eff);
    double* out = kp + (int64_t)cols[0] * h->n_pad;
    if (lists)
      sr_pass_b_kernel<true><<<grid_b, kRows, 0, st>>>(
          p->tiles_s.as<uint8_t>(), h->m_pad / kRows, p->s_ld, planes_b, h->m_pad, sc.sum_c,
          sc.scale_w, sc.scale_c, qc32, p->miss.b_ent.as<uint32_t>(), p->miss.b_seg.as<int64_t>(),
          p->miss.b_nch, p->miss.b_bits, sc.err, out_scale, out);
    else
      sr_pass_b_kernel<false><<<grid_b, kRows, 0, st>>>(
          p->tiles_s.as<uint8_t>(), h->m_pad / kRows, p->s_ld, planes_b, h->m_pad, sc.sum_c,
          sc.scale_w, sc.scale_c, nullptr, nullptr, nullptr, 0, 0, nullptr, out_scale, out);
    SG_CHECK_LAUNCH();
    count_launches(6);
    SG_TRY(mark(&t1));
    if (h->profiling) ev_s.emplace_back(t0, t1);
    h->stats.sc_launches += 1;
    h->stats.sc_list_launches += lists ? 1 : 0;
    h->n_kv += 1;
  }
  for (size_t c0 = 0; c0 < (single ? 0 : cols.size()); c0 += kMaxR) {
    const int r = (int)std::min<size_t>(kMaxR, cols.size() - c0);
    const int ng = (int)round_up(3 * r, 16);
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
                                         p->img_a.as<uint8_t>(), ng, sc.sum_v);
      SG_CHECK_LAUNCH();
    }
    // ---- pass A: u = Z' v ----
    {
      TcArgs a{};
      a.ng = ng;
      a.r = r;
      a.nk = (int)n_stages_a;
      a.tiles = p->tiles_m.as<uint8_t>();
      a.tile_ld = n_stages_a;
      a.img_g = p->img_a.as<uint8_t>();
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
      SG_TRY(launch_tc_tuned<false>(h->device, grid, a, st));
      // leave-one-chromosome-out: the left-out markers' rows of u do not enter pass B
      if (h->masked) SG_CUDA(mask_rows_f64(p->u.as<double>(), h->m_pad, r, h->excl.as<uint8_t>(),
                                           h->m, st));
      SG_TRY(mark(&t1));
      if (h->profiling) ev_a.emplace_back(t0, t1);
      h->stats.tc_pass_a_launches += 1;
      if (p->tracing) SG_TRY(trace_dump(p, "pass A", st));
    }
    // ---- pass B operands ----
    {
      SG_CUDA(cudaMemsetAsync(p->img_w.ptr, 0, (size_t)h->m_pad * ng, st));
      SG_CUDA(cudaMemsetAsync(p->img_c.ptr, 0, (size_t)h->m_pad * ng, st));
      dim3 g1((unsigned)std::min<int64_t>(ceil_div(h->m_pad, 256), 296), (unsigned)r);
      count_launches(2);
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
      a.tiles = p->tiles_s.as<uint8_t>();
      a.tile_ld = p->s_ld;
      a.img_g = p->img_w.as<uint8_t>();
      a.img_m = p->img_c.as<uint8_t>();
      a.scale_g = sc.scale_w;
      a.scale_m = sc.scale_c;
      a.sum_q = reinterpret_cast<const long long*>(sc.sum_c);
      a.out = kp;
      a.out_ld = h->n_pad;
      a.col_map = cmap;
      a.out_scale = 1.0 / (double)(h->masked ? h->m_active : h->m_eff);
      a.err = sc.err;
      a.trace = p->tracing ? p->trace.as<unsigned long long>() : nullptr;
      const unsigned grid = (unsigned)(h->n_pad / kRows);
      cudaEvent_t t0 = nullptr, t1 = nullptr;
      SG_TRY(mark(&t0));
      SG_TRY(launch_tc_tuned<true>(h->device, grid, a, st));
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
  for (auto& pr : ev_s) {
    float ms = 0.f;
    SG_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
    h->stats.sc_ms += ms;
  }
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  if (err & kSrListErr)
    return fail(SAIGE_ECUDA, "one-column GRM product: a missing-call list entry out of range");
  if (err) return fail(SAIGE_TIMEOUT, "tensor-core GRM product: a pipeline wait timed out");
  return Status();
}

}  // namespace saige
