// Device helpers of the hand-written tcgen05 pipelines (the GRM product and the MLP
// of the learned start): mbarriers with bounded waits, bulk copies, shared-memory
// matrix descriptors in the 128-byte swizzle, MMA commits and tensor-memory loads.
// sm_100a only.
#pragma once
#include <stdint.h>

namespace saige {
namespace tcx {

// Budget of a drain wait (work this CTA already issued): ~2 s at 1.9 GHz.
constexpr long long kWaitCycles = 4000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
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

// Non-blocking test of a phase (mbarrier.try_wait may suspend the thread for a while).
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: returns false (and raises the CTA abort flag and the error
// word) when the barrier phase does not complete within `budget` cycles or another
// role already gave up.  A budget of 0 gives up unless the phase has already
// completed (a non-blocking test).
template <bool kBackoff>
__device__ __forceinline__ bool mbar_wait_impl(uint32_t bar, uint32_t parity,
                                               volatile int* abort_flag, unsigned int* err,
                                               long long budget) {
  if (budget <= 0) {
    if (mbar_test_wait(bar, parity)) return true;
    *abort_flag = 1;
    atomicOr(err, 1u);
    return false;
  }
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  uint32_t sleep_ns = 32;
  for (uint32_t polls = 1;; ++polls) {
    if (mbar_try_wait(bar, parity)) return true;
    if (kBackoff) {
      // waiting warps yield their issue slots to the MMA-issuing warp
      __nanosleep(sleep_ns);
      if (sleep_ns < 128) sleep_ns <<= 1;
    }
    if ((polls & 63u) == 0) {  // the clock and the abort flag are checked every 64 polls
      if (*abort_flag) return false;
      if (clock64() - t0 > budget) {
        *abort_flag = 1;
        atomicOr(err, 1u);
        return false;
      }
    }
  }
}

// Wait with exponential back-off (producer, unpack and epilogue warps).
__device__ __forceinline__ bool mbar_wait_sleep(uint32_t bar, uint32_t parity,
                                                volatile int* abort_flag, unsigned int* err,
                                                long long budget) {
  return mbar_wait_impl<true>(bar, parity, abort_flag, err, budget);
}

// Wait for asynchronous work this CTA already issued (its bulk copies, its MMAs),
// which completes whatever the other roles did: the abort flag is not consulted and
// the budget is the fixed one, so that after an abort no copy or MMA is still in
// flight when the CTA frees its TMEM and exits.  False (and the error word) only if
// the hardware does not complete the work within ~2 s.
__device__ __forceinline__ bool mbar_wait_drain(uint32_t bar, uint32_t parity, unsigned int* err) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (uint32_t polls = 1;; ++polls) {
    if (mbar_try_wait(bar, parity)) return true;
    __nanosleep(128);
    if ((polls & 63u) == 0 && clock64() - t0 > kWaitCycles) {
      atomicOr(err, 2u);
      return false;
    }
  }
}

// Non-tensor bulk copy global -> shared (16-byte aligned addresses, size a
// multiple of 16), completing on an mbarrier.  No multicast.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle
// (version 1, sm_100): SBO = 1024 B between 8-row groups, LBO unused (1).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;    // leading byte offset >> 4
  d |= (uint64_t)64u << 32;   // stride byte offset (1024) >> 4
  d |= (uint64_t)1u << 46;    // version
  d |= (uint64_t)2u << 61;    // SWIZZLE_128B
  return d;
}

__device__ __forceinline__ uint4 lds128(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(addr));
  return v;
}

__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ void named_bar_arrive(int id, int nthreads) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
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

__device__ __forceinline__ void tmem_wait_st() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}


}  // namespace tcx
}  // namespace saige
