// The MLP of the learned warm start (16 -> 256 -> 256 -> 256 -> 1, tanh, BF16 weights and
// activations, FP32 arithmetic and master weights).
//
// Examples are (sample, column) pairs e = c * n + i with 16 features F[e*16 .. e*16+16]
// and a target T[e].  Layers: h1 = bf16(tanh(W1 x + b1)), h2 = bf16(tanh(W2 h1 + b2)),
// h3 = bf16(tanh(W3 h2 + b3)), y = w4 . h3 + b4, every parameter used as its BF16 copy.
//
// Forward: the input layer on the CUDA cores writes h1 as a BF16 A-operand image; the
// two 256 x 256 layers run on the tensor cores (tcgen05.mma kind::f16, M = 128 examples,
// N = 256 units, K = 16 per instruction; A tiles streamed by bulk copies through a
// three-slot ring, the layer's weights resident in shared memory, two FP32 accumulators
// in tensor memory so that one tile's epilogue overlaps the next tile's MMAs); their
// epilogues add the bias, apply tanh, round to BF16 and write the next layer's image —
// or, after the last layer, the output y.
//
// Backward (training): the gradient with respect to the FP32 master weights through the
// BF16 roundings (straight through), on the CUDA cores: the output layer elementwise,
// dh = dz W as a blocked FP32 GEMM with the tanh derivative in its epilogue, and the
// weight gradients dW = dz' h as a split-K blocked GEMM whose partials are summed in a
// fixed order, so that training is deterministic.  Adam then updates the master weights
// and their BF16 copy and images; the step loop is captured as a CUDA graph.
#include <cuda_bf16.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <set>
#include <vector>

#include "mlp.cuh"
#include "tcgen05.cuh"

namespace saige {
namespace {

using namespace tcx;

constexpr int H = kMlpH;
constexpr int IN = kMlpIn;
constexpr int kTile = 128;                       // examples per tensor-core tile (MMA M)
constexpr uint32_t kPanelA = kTile * 128;        // 16 KB: 128 rows x 64 BF16 (128 B)
constexpr uint32_t kHalfA = 2 * kPanelA;         // 32 KB: K = 128 of a tile
constexpr uint32_t kTileA = 4 * kPanelA;         // 64 KB: K = 256 of a tile
constexpr uint32_t kPanelW = H * 128;            // 32 KB: 256 rows x 64 BF16
constexpr uint32_t kImgW = 4 * kPanelW;          // 128 KB: one layer's weights
constexpr int kASlots = 3;                       // A ring: K-halves of tiles
constexpr int kLayerThreads = 64 + 32 * 8;       // producer, MMA warp, 8 epilogue warps

__device__ __forceinline__ float bf16_to_f32(uint16_t b) {
  return __uint_as_float((uint32_t)b << 16);
}
__device__ __forceinline__ uint16_t f32_to_bf16(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

// Byte offset of (row r, k) in a K = 256 BF16 operand image of 128-row tiles: four
// 64-column panels per tile, each 128 rows x 128 B in the 128-byte swizzle (16-byte
// chunk j of row r at chunk j ^ (r & 7)) that the shared-memory descriptors expect.
__host__ __device__ __forceinline__ size_t a_img_off(int64_t r, int k) {
  const int64_t t = r / kTile;
  const int rr = (int)(r % kTile);
  const int p = k >> 6, j = (k & 63) >> 3;
  return ((size_t)(t * 4 + p) * kTile + rr) * 128 + (size_t)((j ^ (rr & 7)) << 4) + (k & 7) * 2;
}

// Byte offset of W[n][k] (n < 256 units, k < 256 inputs) in a weight image: panel p
// holds k in [64 p, 64 p + 64) for all 256 rows, in the same swizzle.
__host__ __device__ __forceinline__ size_t w_img_off(int n, int k) {
  const int p = k >> 6, j = (k & 63) >> 3;
  return ((size_t)p * H + n) * 128 + (size_t)((j ^ (n & 7)) << 4) + (k & 7) * 2;
}

// Instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulate,
// M = 128, N = 256.
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(H >> 3) << 17) |
                                ((uint32_t)(kTile >> 4) << 24);

// D[tmem] (+)= A[smem] * B[smem]
__device__ __forceinline__ void mma_bf16_ss(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                            uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdescBf16), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mbar_arrive_local(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Example e of slot s of a pass: the slots of a training step walk the examples with a
// stride coprime with n_ex from the device step counter; otherwise slot s is example
// s0 + s.  Held-out examples (sample index (e % n) % holdout == 0) carry no weight.
struct Walk {
  const int* step;   // training: the device step counter; else NULL
  int64_t per_step;  // training: examples per step
  int64_t stride;    // training: the walk's multiplier
  int64_t s0;        // inference: first example of the chunk
  int64_t n_ex, n;
  int holdout;       // > 0: drop held-out examples (training) or visit only them (validation)
  int held_only;     // 1: slot s is the s-th held-out example (validation)
};

__device__ __forceinline__ int64_t walk_example(const Walk& w, int64_t s) {
  if (w.step) {
    const unsigned long long g = (unsigned long long)(*w.step) * (unsigned long long)w.per_step +
                                 (unsigned long long)s;
    return (int64_t)((g * (unsigned long long)w.stride) % (unsigned long long)w.n_ex);
  }
  if (w.held_only) {
    const int64_t nh = (w.n + w.holdout - 1) / w.holdout;
    const int64_t j = w.s0 + s;
    return (j / nh) * w.n + (j % nh) * w.holdout;
  }
  return w.s0 + s;
}

// Input layer on the CUDA cores: thread = one row of the chunk (rows past `rows` are
// written as the image's zero padding).  Writes h1 as BF16 into the A image, and for
// training the gathered features x (FP32), the unrounded h1 (FP32), the target and the
// example's weight (0 for held-out examples).
__global__ void __launch_bounds__(128)
    mlp_input_kernel(const uint16_t* __restrict__ wbf, const float* __restrict__ F,
                     const float* __restrict__ Tg, Walk walk, int64_t rows,
                     uint8_t* __restrict__ img1, float* __restrict__ xb, float* __restrict__ h1,
                     float* __restrict__ tb, float* __restrict__ mb) {
  __shared__ float w1[H * IN];
  __shared__ float b1[H];
  for (int t = threadIdx.x; t < H * IN; t += blockDim.x) w1[t] = bf16_to_f32(wbf[kMlpW1 + t]);
  for (int t = threadIdx.x; t < H; t += blockDim.x) b1[t] = bf16_to_f32(wbf[kMlpB1 + t]);
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float x[IN];
#pragma unroll
  for (int k = 0; k < IN; ++k) x[k] = 0.f;
  bool live = r < rows;
  int64_t e = 0;
  if (live) {
    e = walk_example(walk, r);
    const float4* src = reinterpret_cast<const float4*>(F + e * IN);
#pragma unroll
    for (int q = 0; q < IN / 4; ++q) {
      const float4 v = src[q];
      x[4 * q] = v.x; x[4 * q + 1] = v.y; x[4 * q + 2] = v.z; x[4 * q + 3] = v.w;
    }
    if (xb) {
#pragma unroll
      for (int k = 0; k < IN; ++k) xb[r * IN + k] = x[k];
    }
    if (tb) {
      bool use = true;
      if (walk.step && walk.holdout > 0 && ((e % walk.n) % walk.holdout) == 0) use = false;
      tb[r] = Tg[e];
      mb[r] = use ? 1.f : 0.f;
    }
  }
  for (int j0 = 0; j0 < H; j0 += 8) {
    uint32_t packed[4];
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
      float hv[2];
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        const int j = j0 + u + v;
        float z = b1[j];
#pragma unroll
        for (int k = 0; k < IN; ++k) z = fmaf(w1[j * IN + k], x[k], z);
        const float h = live ? tanhf(z) : 0.f;
        if (h1 && live) h1[r * H + j] = h;
        hv[v] = h;
      }
      packed[u >> 1] = (uint32_t)f32_to_bf16(hv[0]) | ((uint32_t)f32_to_bf16(hv[1]) << 16);
    }
    *reinterpret_cast<uint4*>(img1 + a_img_off(r, j0)) =
        make_uint4(packed[0], packed[1], packed[2], packed[3]);
  }
}

// ---------------------------------------------------------------------------
// A 256 x 256 layer on the tensor cores
// ---------------------------------------------------------------------------
struct LayerArgs {
  const uint8_t* a_img;   // input activations: `tiles` tiles of 64 KB (a_img_off)
  const uint8_t* w_img;   // the layer's weights, 128 KB (w_img_off)
  const uint16_t* wbf;    // BF16 parameters (bias; w4 and b4 for the output)
  int b_off;              // kMlpB2 or kMlpB3
  int64_t rows;           // valid rows (examples) of the chunk
  int64_t tiles;          // ceil(rows / 128)
  uint8_t* out_img;       // hidden layer: the next layer's image (every row of every tile)
  float* hbuf;            // optional: unrounded tanh activations, rows x 256 FP32
  float* y;               // output layer: rows outputs
  long long wait_cycles;  // budget of each pipeline wait
  unsigned int* err;      // bit 0: a wait ran out; bit 1: a drain ran out
};

// Shared memory: W (128 KB) | A ring (3 x 32 KB) | 14 barriers | TMEM address, abort
// flag | y partials [2][128] (output layer).
constexpr uint32_t kLayerBars = kImgW + kASlots * kHalfA;
constexpr uint32_t kLayerSmem = 1024 + kLayerBars + 128 + 2 * kTile * 4;

// Thread roles: warp 0 streams the A tiles (K-halves) through the ring, warp 1 issues
// the MMAs (lane 0) of each tile into accumulator (tile & 1), warps 2-9 run the epilogue,
// two warps per TMEM lane group (warp % 4), each over 128 of the 256 units.  Every wait
// is bounded; after an abort no MMA is issued, and before the tensor memory is freed the
// MMA warp's final commit and the producer's copies are waited for.
template <bool kLast>
__global__ void __launch_bounds__(kLayerThreads, 1) mlp_layer_kernel(LayerArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gen = smem_raw + (base - raw);
  const uint32_t sW = base, sA = base + kImgW, bars = base + kLayerBars;
  auto WFULL = [&]() { return bars; };
  auto AFULL = [&](int s) { return bars + 8u + 8u * s; };
  auto AEMPTY = [&](int s) { return bars + 32u + 8u * s; };
  auto DFULL = [&](int d) { return bars + 56u + 8u * d; };
  auto DEMPTY = [&](int d) { return bars + 72u + 8u * d; };
  auto YREADY = [&](int d) { return bars + 88u + 8u * d; };
  const uint32_t FIN = bars + 104u;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gen + kLayerBars + 112);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gen + kLayerBars + 116);
  float* ypart = reinterpret_cast<float*>(gen + kLayerBars + 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t n_my = a.tiles > blockIdx.x ? (a.tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (threadIdx.x == 0) {
    mbar_init(WFULL(), 1);
    for (int s = 0; s < kASlots; ++s) {
      mbar_init(AFULL(s), 1);
      mbar_init(AEMPTY(s), 1);
    }
    for (int d = 0; d < 2; ++d) {
      mbar_init(DFULL(d), 1);
      mbar_init(DEMPTY(d), 8);
      mbar_init(YREADY(d), 4);
    }
    mbar_init(FIN, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      mbar_expect_tx(WFULL(), kImgW);
      for (int p = 0; p < 4; ++p)
        bulk_load(sW + p * kPanelW, a.w_img + (size_t)p * kPanelW, kPanelW, WFULL());
      int S = 0, issued = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int64_t i = 0; i < n_my && ok; ++i) {
        const int64_t t = blockIdx.x + i * gridDim.x;
        for (int h = 0; h < 2; ++h) {
          const int J = (int)(2 * i + h);
          if (J >= kASlots &&
              !mbar_wait_sleep(AEMPTY(S), ph ^ 1u, abort_flag, a.err, a.wait_cycles)) {
            ok = false;
            break;
          }
          mbar_expect_tx(AFULL(S), kHalfA);
          bulk_load(sA + S * kHalfA, a.a_img + (size_t)t * kTileA + (size_t)h * kHalfA, kHalfA,
                    AFULL(S));
          issued = J + 1;
          if (++S == kASlots) { S = 0; ph ^= 1u; }
        }
      }
      // every issued copy has landed before the CTA exits (only the last kASlots A
      // loads can still be in flight: load J was issued after load J - kASlots was
      // consumed)
      for (int J = issued > kASlots ? issued - kASlots : 0; J < issued; ++J)
        mbar_wait_drain(AFULL(J % kASlots), (uint32_t)((J / kASlots) & 1), a.err);
      mbar_wait_drain(WFULL(), 0u, a.err);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    int ok = lane == 0 ? (int)mbar_wait_sleep(WFULL(), 0u, abort_flag, a.err, a.wait_cycles) : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    int S = 0;
    uint32_t ph = 0;
    // (lane 0) the last A half and the last tile whose AEMPTY / DFULL was committed
    int64_t j_done = -1, i_done = -1;
    for (int64_t i = 0; i < n_my && ok; ++i) {
      const int d = (int)(i & 1);
      if (i >= 2) {
        int w = lane == 0 ? (int)mbar_wait_sleep(DEMPTY(d), (uint32_t)(((i >> 1) - 1) & 1),
                                                 abort_flag, a.err, a.wait_cycles)
                          : 0;
        ok = __shfl_sync(0xffffffffu, w, 0);
        if (!ok) break;
      }
      for (int h = 0; h < 2; ++h) {
        int w = lane == 0 ? (int)mbar_wait_sleep(AFULL(S), ph, abort_flag, a.err, a.wait_cycles)
                          : 0;
        ok = __shfl_sync(0xffffffffu, w, 0);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (lane == 0) {
#pragma unroll
          for (int pp = 0; pp < 2; ++pp) {
            const uint64_t ad = sw128_desc(sA + S * kHalfA + pp * kPanelA);
            const uint64_t bd = sw128_desc(sW + (2 * h + pp) * kPanelW);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)  // K = 16 BF16 = 32 bytes per instruction
              mma_bf16_ss(tmem + (uint32_t)d * H, ad + 2u * kk, bd + 2u * kk,
                          (h | pp | kk) != 0 ? 1u : 0u);
          }
          mma_commit(AEMPTY(S));
          j_done = 2 * i + h;
        }
        if (++S == kASlots) { S = 0; ph ^= 1u; }
      }
      if (!ok) break;
      if (lane == 0) {
        mma_commit(DFULL(d));
        i_done = i;
      }
    }
    __syncwarp();
    if (lane == 0) {
      mma_commit(FIN);
      // A commit's arrival is performed when its MMAs complete, in no set order with the
      // other commits: wait for the last committed phase of every slot and accumulator
      // barrier, so that none lands in the shared memory of the next CTA on this SM.
      mbar_wait_drain(FIN, 0u, a.err);
      for (int sl = 0; sl < kASlots; ++sl) {
        if (j_done < sl) continue;
        const int64_t j = j_done - (j_done - sl) % kASlots;
        mbar_wait_drain(AEMPTY(sl), (uint32_t)((j / kASlots) & 1), a.err);
      }
      for (int dd = 0; dd < 2; ++dd) {
        if (i_done < dd) continue;
        const int64_t ii = i_done - (i_done - dd) % 2;
        mbar_wait_drain(DFULL(dd), (uint32_t)((ii >> 1) & 1), a.err);
      }
    }
  } else {
    // ---------------- epilogue ----------------
    const int ew = warp - 2, lg = warp & 3, ch = ew >> 2;
    const int row = lg * 32 + lane;
    const uint32_t lane_off = (uint32_t)(lg * 32) << 16;
    const float b4 = kLast ? bf16_to_f32(a.wbf[kMlpB4]) : 0.f;
    for (int64_t i = 0; i < n_my; ++i) {
      const int d = (int)(i & 1);
      bool ok = mbar_wait_sleep(DFULL(d), (uint32_t)((i >> 1) & 1), abort_flag, a.err,
                                a.wait_cycles);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int64_t t = blockIdx.x + i * gridDim.x;
      const int64_t r = t * kTile + row;
      const bool in = r < a.rows;
      float ysum = 0.f;
#pragma unroll 1
      for (int c0 = ch * 128; c0 < ch * 128 + 128; c0 += 16) {
        uint32_t v[16];
        tmem_ld16(tmem + (uint32_t)d * H + lane_off + (uint32_t)c0, v);
        tmem_wait_ld();
        uint32_t packed[8];
#pragma unroll
        for (int u = 0; u < 16; u += 2) {
          float hb[2];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int c = c0 + u + q;
            const float z = __uint_as_float(v[u + q]) + bf16_to_f32(a.wbf[a.b_off + c]);
            const float h = tanhf(z);
            if (a.hbuf && in) a.hbuf[r * H + c] = h;
            hb[q] = bf16_to_f32(f32_to_bf16(h));
            if (kLast) ysum = fmaf(bf16_to_f32(a.wbf[kMlpW4 + c]), hb[q], ysum);
          }
          packed[u >> 1] = (uint32_t)f32_to_bf16(hb[0]) | ((uint32_t)f32_to_bf16(hb[1]) << 16);
        }
        if (!kLast) {
          *reinterpret_cast<uint4*>(a.out_img + a_img_off(r, c0)) =
              make_uint4(packed[0], packed[1], packed[2], packed[3]);
          *reinterpret_cast<uint4*>(a.out_img + a_img_off(r, c0 + 8)) =
              make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
      }
      if (kLast) {
        // the second half of the units hands its partial sum to the first
        if (ch == 1) {
          ypart[d * kTile + row] = ysum;
          __syncwarp();
          if (lane == 0) mbar_arrive_local(YREADY(d));
        } else {
          const bool yk = mbar_wait_sleep(YREADY(d), (uint32_t)((i >> 1) & 1), abort_flag, a.err,
                                          a.wait_cycles);
          if (yk && in) a.y[r] = ysum + ypart[d * kTile + row] + b4;
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive_local(DEMPTY(d));
    }
  }

  __syncwarp();
  if (warp == 1) mbar_wait_drain(FIN, 0u, a.err);  // no MMA in flight past this point
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
  }
}

// ---------------------------------------------------------------------------
// Backward pass and optimiser (CUDA cores, FP32, fixed summation orders)
// ---------------------------------------------------------------------------
// Output layer: gy = 2 (y - t) m scale (m = the example's weight); dz3 = gy w4 (1 - h3^2);
// the summed squared error into sep (one partial per block, summed in order later).
__global__ void mlp_out_grad_kernel(const uint16_t* __restrict__ wbf, const float* __restrict__ y,
                                    const float* __restrict__ tb, const float* __restrict__ mb,
                                    const float* __restrict__ h3, float scale,
                                    float* __restrict__ gy, float* __restrict__ dz3,
                                    double* __restrict__ sep) {
  const int64_t r = blockIdx.x;  // one block of 256 threads per row
  const int j = threadIdx.x;
  const float err = (y[r] - tb[r]) * mb[r];
  const float g = 2.f * err * scale;
  const float h = h3[r * H + j];
  dz3[r * H + j] = g * bf16_to_f32(wbf[kMlpW4 + j]) * (1.f - h * h);
  if (j == 0) {
    gy[r] = g;
    sep[r] = (double)err * (double)err;
  }
}

// C[r][k] = (sum_j dz[r][j] W[j][k]) (1 - h[r][k]^2): the gradient through layer l's
// weights back to the previous layer's pre-activation.  64 x 64 tiles, 256 threads of
// 4 x 4 outputs, j in steps of 16 through shared memory; W from its BF16 copy.
__global__ void __launch_bounds__(256)
    mlp_back_kernel(const float* __restrict__ dz, const uint16_t* __restrict__ wbf, int w_off,
                    const float* __restrict__ h, int64_t rows, float* __restrict__ out) {
  __shared__ float As[16][64 + 4];
  __shared__ float Bs[16][64 + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int64_t r0 = (int64_t)blockIdx.x * 64;
  const int k0 = blockIdx.y * 64;
  float acc[4][4] = {};
  for (int j0 = 0; j0 < H; j0 += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int jj = t & 15, rr = t >> 4;
      const int64_t r = r0 + rr;
      As[jj][rr] = r < rows ? dz[r * H + j0 + jj] : 0.f;
      const int kk = t & 63, j2 = t >> 6;
      Bs[j2][kk] = bf16_to_f32(wbf[w_off + (j0 + j2) * H + k0 + kk]);
    }
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < 16; ++jj) {
      float av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        av[u] = As[jj][ty * 4 + u];
        bv[u] = Bs[jj][tx * 4 + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int64_t r = r0 + ty * 4 + u;
    if (r >= rows) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int k = k0 + tx * 4 + v;
      const float hv = h[r * H + k];
      out[r * H + k] = acc[u][v] * (1.f - hv * hv);
    }
  }
}

// Split-K weight gradient: part[s][j][k] = sum over rows r of split s of dz[r][j] a[r][k],
// a the layer's input (BF16-rounded when round_a: the values the forward pass used;
// width kin = 256, or 16 for the input layer), plus bias partials (k == kin column:
// sum of dz) when bias.  Splits of kSplitRows rows; 64 x 64 output tiles.
constexpr int kSplitRows = 512;

__global__ void __launch_bounds__(256)
    mlp_wgrad_kernel(const float* __restrict__ dz, const float* __restrict__ a, int kin,
                     int round_a, int64_t rows, float* __restrict__ part, int ldp) {
  __shared__ float As[16][64 + 4];
  __shared__ float Bs[16][64 + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int j0 = blockIdx.x * 64, k0 = blockIdx.y * 64;
  const int64_t s = blockIdx.z;
  const int64_t rb = s * kSplitRows, re = std::min<int64_t>(rows, rb + kSplitRows);
  float acc[4][4] = {};
  for (int64_t e0 = rb; e0 < re; e0 += 16) {
    for (int t = threadIdx.x; t < 16 * 64; t += 256) {
      const int ee = t >> 6, c = t & 63;
      const int64_t e = e0 + ee;
      As[ee][c] = e < re ? dz[e * H + j0 + c] : 0.f;
      float av = 0.f;
      if (e < re && k0 + c < kin) {
        av = a[e * kin + k0 + c];
        if (round_a) av = bf16_to_f32(f32_to_bf16(av));
      } else if (e < re && k0 + c == kin) {
        av = 1.f;  // the bias column
      }
      Bs[ee][c] = av;
    }
    __syncthreads();
#pragma unroll
    for (int ee = 0; ee < 16; ++ee) {
      float av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        av[u] = As[ee][ty * 4 + u];
        bv[u] = Bs[ee][tx * 4 + u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(av[u], bv[v], acc[u][v]);
    }
    __syncthreads();
  }
  float* P = part + s * (int64_t)H * ldp;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int k = k0 + tx * 4 + v;
      if (k <= kin) P[(j0 + ty * 4 + u) * ldp + k] = acc[u][v];
    }
}

// grad[w_off + j*kin + k] = sum_s part[s][j][k] (k < kin), grad[b_off + j] = sum_s
// part[s][j][kin]; in split order.
__global__ void mlp_wgrad_sum_kernel(const float* __restrict__ part, int nsplit, int kin, int ldp,
                                     float* __restrict__ grad, int w_off, int b_off) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= H * (kin + 1)) return;
  const int j = idx / (kin + 1), k = idx % (kin + 1);
  float sacc = 0.f;
  for (int s = 0; s < nsplit; ++s) sacc += part[(int64_t)s * H * ldp + j * ldp + k];
  if (k < kin) grad[w_off + j * kin + k] = sacc;
  else grad[b_off + j] = sacc;
}

// Output weights: grad[w4 + j] = sum_r gy[r] bf16(h3[r][j]), grad[b4] = sum_r gy[r], and
// the loss: sum of sep; each thread one column, rows in order.
__global__ void mlp_out_sum_kernel(const float* __restrict__ gy, const float* __restrict__ h3,
                                   const double* __restrict__ sep, int64_t rows,
                                   float* __restrict__ grad, double* __restrict__ loss) {
  const int j = threadIdx.x;
  if (j < H) {
    float s = 0.f;
    for (int64_t r = 0; r < rows; ++r) s = fmaf(gy[r], bf16_to_f32(f32_to_bf16(h3[r * H + j])), s);
    grad[kMlpW4 + j] = s;
  } else if (j == H) {
    float s = 0.f;
    for (int64_t r = 0; r < rows; ++r) s += gy[r];
    grad[kMlpB4] = s;
  } else if (j == H + 1) {
    double s = 0.0;
    for (int64_t r = 0; r < rows; ++r) s += sep[r];
    loss[0] = s;
    loss[1] = (double)rows;
  }
}

// Adam (Kingma and Ba, 2015); then the BF16 copy.
__global__ void mlp_adam_kernel(const float* __restrict__ g, float* __restrict__ w,
                                uint16_t* __restrict__ wbf, float* __restrict__ m1,
                                float* __restrict__ m2, const int* __restrict__ step, float lr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kMlpParams) return;
  const int s = *step + 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float gv = g[p];
  const float mm = b1 * m1[p] + (1.f - b1) * gv;
  const float vv = b2 * m2[p] + (1.f - b2) * gv * gv;
  m1[p] = mm;
  m2[p] = vv;
  const float mh = mm / (1.f - powf(b1, (float)s));
  const float vh = vv / (1.f - powf(b2, (float)s));
  const float nw = w[p] - lr * mh / (sqrtf(vh) + 1e-8f);
  w[p] = nw;
  wbf[p] = f32_to_bf16(nw);
}

__global__ void mlp_step_kernel(int* step) { *step += 1; }

__global__ void mlp_to_bf16_kernel(const float* __restrict__ w, uint16_t* __restrict__ wbf) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) wbf[p] = f32_to_bf16(w[p]);
}

// The B-operand images of W2 and W3 from the BF16 copy: one thread per 8 inputs of a row.
__global__ void mlp_wimage_kernel(const uint16_t* __restrict__ wbf, uint8_t* __restrict__ img) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // 2 layers x 256 rows x 32 groups
  if (idx >= 2 * H * (H / 8)) return;
  const int l = idx / (H * (H / 8)), rem = idx % (H * (H / 8));
  const int n = rem / (H / 8), k0 = (rem % (H / 8)) * 8;
  const uint16_t* w = wbf + (l == 0 ? kMlpW2 : kMlpW3) + n * H + k0;
  uint32_t p[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) p[u] = (uint32_t)w[2 * u] | ((uint32_t)w[2 * u + 1] << 16);
  *reinterpret_cast<uint4*>(img + (size_t)l * kImgW + w_img_off(n, k0)) =
      make_uint4(p[0], p[1], p[2], p[3]);
}

// Held-out squared error and squared target over y[j] (held-out example j) — partials
// per block.
__global__ void mlp_val_kernel(const float* __restrict__ y, const float* __restrict__ Tg, Walk walk,
                               int64_t n_out, double* __restrict__ part) {
  __shared__ double sh[2][8];
  double se = 0.0, st = 0.0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_out;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = walk_example(walk, j);
    const double d = (double)y[j] - (double)Tg[e];
    se += d * d;
    st += (double)Tg[e] * (double)Tg[e];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    se += __shfl_xor_sync(0xffffffffu, se, o);
    st += __shfl_xor_sync(0xffffffffu, st, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = se;
    sh[1][threadIdx.x >> 5] = st;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      a += sh[0][i];
      b += sh[1][i];
    }
    part[2 * blockIdx.x] = a;
    part[2 * blockIdx.x + 1] = b;
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
constexpr int64_t kChunkRows = 131072;  // examples per inference chunk (2 x 64 MB of images)
constexpr int kGraphSteps = 25;

int64_t round_tile(int64_t r) { return (r + kTile - 1) / kTile * kTile; }

struct Work {
  uint8_t *img1 = nullptr, *img2 = nullptr;
  float *y = nullptr, *xb = nullptr, *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
  float *tb = nullptr, *mb = nullptr, *gy = nullptr, *dza = nullptr, *dzb = nullptr;
  double* sep = nullptr;
};

size_t work_bytes(int64_t rows, bool train) {
  size_t b = (size_t)rows * (2 * 512 + 4);
  if (train) b += (size_t)rows * (IN * 4 + 5 * H * 4 + 3 * 4 + 8);
  return b + 256;
}

Status mlp_work(Mlp& m, int64_t rows, bool train, Work& w) {
  rows = round_tile(rows);
  SG_TRY(m.work.reserve(work_bytes(rows, train)));
  char* p = m.work.as<char>();
  auto take = [&](size_t bytes) {
    char* q = p;
    p += (bytes + 255) & ~(size_t)255;
    return q;
  };
  w.img1 = reinterpret_cast<uint8_t*>(take((size_t)rows * 512));
  w.img2 = reinterpret_cast<uint8_t*>(take((size_t)rows * 512));
  w.y = reinterpret_cast<float*>(take((size_t)rows * 4));
  if (train) {
    w.xb = reinterpret_cast<float*>(take((size_t)rows * IN * 4));
    w.h1 = reinterpret_cast<float*>(take((size_t)rows * H * 4));
    w.h2 = reinterpret_cast<float*>(take((size_t)rows * H * 4));
    w.h3 = reinterpret_cast<float*>(take((size_t)rows * H * 4));
    w.dza = reinterpret_cast<float*>(take((size_t)rows * H * 4));
    w.dzb = reinterpret_cast<float*>(take((size_t)rows * H * 4));
    w.tb = reinterpret_cast<float*>(take((size_t)rows * 4));
    w.mb = reinterpret_cast<float*>(take((size_t)rows * 4));
    w.gy = reinterpret_cast<float*>(take((size_t)rows * 4));
    w.sep = reinterpret_cast<double*>(take((size_t)rows * 8));
  }
  return Status();
}

// The dynamic shared-memory limit of the layer kernels is a per-device attribute.
cudaError_t set_smem_attrs(int* sms) {
  static std::mutex mu;
  static std::set<int> done;
  static int sm_count[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (!done.count(dev)) {
    e = cudaFuncSetAttribute(mlp_layer_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kLayerSmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(mlp_layer_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kLayerSmem);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sm_count[dev & 63], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    done.insert(dev);
  }
  *sms = sm_count[dev & 63];
  return cudaSuccess;
}

// The forward pass of `rows` examples of the walk; with train, the activations, the
// gathered features, the targets and the example weights for the backward pass.
Status forward_rows(Mlp& m, const float* F, const float* T, const Walk& walk, int64_t rows,
                    const Work& w, bool train, float* yout, cudaStream_t st) {
  int sms = 148;
  SG_CUDA(set_smem_attrs(&sms));
  const int64_t tiles = round_tile(rows) / kTile;
  mlp_input_kernel<<<(unsigned)tiles, kTile, 0, st>>>(m.wbf, F, T, walk, rows, w.img1,
                                                      train ? w.xb : nullptr,
                                                      train ? w.h1 : nullptr,
                                                      train ? w.tb : nullptr,
                                                      train ? w.mb : nullptr);
  LayerArgs a{};
  a.wbf = m.wbf;
  a.rows = rows;
  a.tiles = tiles;
  a.wait_cycles = kWaitCycles;
  a.err = m.err;
  const unsigned grid = (unsigned)std::min<int64_t>(tiles, sms);
  a.a_img = w.img1;
  a.w_img = m.wimg.as<uint8_t>();
  a.b_off = kMlpB2;
  a.out_img = w.img2;
  a.hbuf = train ? w.h2 : nullptr;
  mlp_layer_kernel<false><<<grid, kLayerThreads, kLayerSmem, st>>>(a);
  a.a_img = w.img2;
  a.w_img = m.wimg.as<uint8_t>() + kImgW;
  a.b_off = kMlpB3;
  a.out_img = nullptr;
  a.hbuf = train ? w.h3 : nullptr;
  a.y = yout;
  mlp_layer_kernel<true><<<grid, kLayerThreads, kLayerSmem, st>>>(a);
  count_launches(3);
  return Status();
}

// One weight-gradient GEMM and its ordered sum into m.grad.
Status wgrad(Mlp& m, const float* dz, const float* a, int kin, bool round_a, int64_t rows,
             int w_off, int b_off, cudaStream_t st) {
  const int ldp = kin + 1;
  const int nsplit = (int)std::max<int64_t>(1, (rows + kSplitRows - 1) / kSplitRows);
  SG_TRY(m.gpart.reserve((size_t)nsplit * H * ldp * sizeof(float)));
  mlp_wgrad_kernel<<<dim3(H / 64, (unsigned)((kin + 1 + 63) / 64), (unsigned)nsplit), 256, 0, st>>>(
      dz, a, kin, round_a ? 1 : 0, rows, m.gpart.as<float>(), ldp);
  mlp_wgrad_sum_kernel<<<(unsigned)((H * (kin + 1) + 255) / 256), 256, 0, st>>>(
      m.gpart.as<float>(), nsplit, kin, ldp, m.grad, w_off, b_off);
  count_launches(2);
  return Status();
}

// m.grad and m.loss from the activations of the last training forward pass.
Status backward_rows(Mlp& m, const Work& w, int64_t rows, float scale, cudaStream_t st) {
  mlp_out_grad_kernel<<<(unsigned)rows, H, 0, st>>>(m.wbf, w.y, w.tb, w.mb, w.h3, scale, w.gy,
                                                    w.dza, w.sep);
  mlp_out_sum_kernel<<<1, H + 32, 0, st>>>(w.gy, w.h3, w.sep, rows, m.grad, m.loss);
  count_launches(2);
  SG_TRY(wgrad(m, w.dza, w.h2, H, true, rows, kMlpW3, kMlpB3, st));
  const dim3 gb((unsigned)((rows + 63) / 64), H / 64);
  mlp_back_kernel<<<gb, 256, 0, st>>>(w.dza, m.wbf, kMlpW3, w.h2, rows, w.dzb);
  count_launches(1);
  SG_TRY(wgrad(m, w.dzb, w.h1, H, true, rows, kMlpW2, kMlpB2, st));
  mlp_back_kernel<<<gb, 256, 0, st>>>(w.dzb, m.wbf, kMlpW2, w.h1, rows, w.dza);
  count_launches(1);
  SG_TRY(wgrad(m, w.dza, w.xb, IN, false, rows, kMlpW1, kMlpB1, st));
  SG_CHECK_LAUNCH();
  return Status();
}

// A multiplier coprime with n_ex for the mini-batch walk.
int64_t batch_stride(int64_t n_ex) {
  static const int64_t primes[] = {2654435761LL, 2246822519LL, 3266489917LL, 668265263LL,
                                   374761393LL};
  for (int64_t p : primes) {
    int64_t a = p % n_ex, b = n_ex;
    while (b) {
      const int64_t t = a % b;
      a = b;
      b = t;
    }
    if (a == 1) return p % n_ex == 0 ? 1 : p % n_ex;
  }
  return 1;
}

Status check_err(Mlp& m, cudaStream_t st) {
  unsigned int e = 0;
  SG_CUDA(cudaMemcpyAsync(&e, m.err, sizeof(e), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (e) return fail(SAIGE_TIMEOUT, "MLP tensor-core layer: a pipeline wait timed out");
  return Status();
}

}  // namespace

void mlp_initial_weights(uint64_t seed, std::vector<float>& w) {
  const size_t nf = (size_t)kMlpParams;
  // uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a splitmix64 stream
  w.assign(nf, 0.f);
  uint64_t x = seed;
  auto uni = [&x]() {
    x += 0x9E3779B97F4A7C15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int count, int fan_in) {
    const double r = 1.0 / std::sqrt((double)fan_in);
    for (int i = 0; i < count; ++i) w[(size_t)off + i] = (float)((2.0 * uni() - 1.0) * r);
  };
  fill(kMlpW1, H * IN, IN);
  fill(kMlpB1, H, IN);
  fill(kMlpW2, H * H, H);
  fill(kMlpB2, H, H);
  fill(kMlpW3, H * H, H);
  fill(kMlpB3, H, H);
  fill(kMlpW4, H, H);
  fill(kMlpB4, 1, H);
}

Status mlp_alloc(Mlp& m) {
  const size_t nf = (size_t)kMlpParams;
  SG_TRY(m.mem.reserve(nf * 4 * 4 + nf * 2 + 256));
  char* b = m.mem.as<char>();
  m.master = reinterpret_cast<float*>(b);
  m.grad = m.master + nf;
  m.m1 = m.grad + nf;
  m.m2 = m.m1 + nf;
  m.loss = reinterpret_cast<double*>(m.m2 + nf);
  m.step = reinterpret_cast<int*>(m.loss + 2);
  m.err = reinterpret_cast<unsigned int*>(m.step + 4);
  m.wbf = reinterpret_cast<uint16_t*>(m.err + 4);
  SG_TRY(m.wimg.reserve(2 * (size_t)kImgW));
  return Status();
}

Status mlp_set(Mlp& m, const float* host_w, cudaStream_t st) {
  const size_t nf = (size_t)kMlpParams;
  SG_CUDA(cudaMemcpyAsync(m.master, host_w, nf * 4, cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemsetAsync(m.m1, 0, nf * 4 * 2, st));
  SG_CUDA(cudaMemsetAsync(m.step, 0, 8 * sizeof(int), st));  // step and err
  mlp_to_bf16_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(m.master, m.wbf);
  mlp_wimage_kernel<<<(2 * H * (H / 8) + 255) / 256, 256, 0, st>>>(m.wbf, m.wimg.as<uint8_t>());
  count_launches(2);
  SG_CHECK_LAUNCH();
  m.ready = true;
  m.trained_steps = 0;
  return Status();
}

Status mlp_init(Mlp& m, uint64_t seed, cudaStream_t st) {
  std::vector<float> w;
  mlp_initial_weights(seed, w);
  SG_TRY(mlp_alloc(m));
  SG_TRY(mlp_set(m, w.data(), st));
  SG_CUDA(cudaStreamSynchronize(st));  // w is a host temporary
  return Status();
}

Status mlp_forward(Mlp& m, const float* F, int64_t n_ex, float* out, cudaStream_t st) {
  if (n_ex <= 0) return Status();
  Work w;
  const int64_t chunk = std::min<int64_t>(n_ex, kChunkRows);
  SG_TRY(mlp_work(m, chunk, false, w));
  for (int64_t s0 = 0; s0 < n_ex; s0 += chunk) {
    Walk walk{nullptr, 0, 0, s0, n_ex, n_ex, 0, 0};
    SG_TRY(forward_rows(m, F, nullptr, walk, std::min<int64_t>(chunk, n_ex - s0), w, false,
                        out + s0, st));
  }
  SG_CHECK_LAUNCH();
  return Status();
}

Status mlp_grad(Mlp& m, const float* F, const float* T, int64_t n_ex, cudaStream_t st) {
  if (n_ex <= 0) return fail(SAIGE_EINVAL, "no examples");
  Work w;
  SG_TRY(mlp_work(m, n_ex, true, w));
  Walk walk{nullptr, 0, 0, 0, n_ex, n_ex, 0, 0};
  SG_TRY(forward_rows(m, F, T, walk, n_ex, w, true, w.y, st));
  SG_TRY(backward_rows(m, w, n_ex, 1.0f / (float)n_ex, st));
  return check_err(m, st);
}

Status mlp_train(Mlp& m, const float* F, const float* T, int64_t n, int q, int steps, float lr,
                 int holdout, cudaStream_t st) {
  if (steps <= 0) return Status();
  const int64_t n_ex = n * q;
  const int per = std::min(steps, kGraphSteps);
  const bool same = m.graph && m.graph_key[0] == F && m.graph_key[1] == T && m.graph_n == n &&
                    m.graph_q == q && m.graph_holdout == holdout && m.graph_lr == lr &&
                    m.graph_steps == per;
  if (!same) {
    if (m.graph) {
      cudaGraphExecDestroy(m.graph);
      m.graph = nullptr;
    }
    Work w;
    SG_TRY(mlp_work(m, kMlpBatch, true, w));
    SG_TRY(m.gpart.reserve((size_t)(kMlpBatch / kSplitRows) * H * (H + 1) * sizeof(float)));
    int sms = 148;
    SG_CUDA(set_smem_attrs(&sms));
    const Walk walk{m.step, kMlpBatch, batch_stride(n_ex), 0, n_ex, n, holdout, 0};
    // the step loop as one graph: forward, backward, Adam, the weight images, the step
    cudaGraph_t graph = nullptr;
    SG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    Status cs;
    for (int s = 0; s < per && cs.ok(); ++s) {
      cs = forward_rows(m, F, T, walk, kMlpBatch, w, true, w.y, st);
      if (cs.ok()) cs = backward_rows(m, w, kMlpBatch, 1.0f / (float)kMlpBatch, st);
      if (!cs.ok()) break;
      mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(m.grad, m.master, m.wbf, m.m1,
                                                               m.m2, m.step, lr);
      mlp_wimage_kernel<<<(2 * H * (H / 8) + 255) / 256, 256, 0, st>>>(m.wbf,
                                                                      m.wimg.as<uint8_t>());
      mlp_step_kernel<<<1, 1, 0, st>>>(m.step);
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (!cs.ok()) {
      if (graph) cudaGraphDestroy(graph);
      return cs;
    }
    if (ce != cudaSuccess)
      return fail(SAIGE_ECUDA, "graph capture failed: %s", cudaGetErrorString(ce));
    const cudaError_t ie = cudaGraphInstantiate(&m.graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      m.graph = nullptr;
      return fail(SAIGE_ECUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
    }
    m.graph_key[0] = F;
    m.graph_key[1] = T;
    m.graph_n = n;
    m.graph_q = q;
    m.graph_holdout = holdout;
    m.graph_lr = lr;
    m.graph_steps = per;
  }
  const int launches = (steps + per - 1) / per;
  for (int l = 0; l < launches; ++l) SG_CUDA(cudaGraphLaunch(m.graph, st));
  count_launches(3 * per * launches);
  m.trained_steps += (int64_t)per * launches;
  return Status();
}

Status mlp_validate(Mlp& m, const float* F, const float* T, int64_t n, int q, int holdout,
                    double* mse, double* target_ms, cudaStream_t st) {
  const int64_t nh = (n + holdout - 1) / holdout, n_out = nh * q;
  if (n_out <= 0) {
    *mse = *target_ms = 0.0;
    return Status();
  }
  DevBuf y, part;
  SG_TRY(y.reserve((size_t)n_out * sizeof(float)));
  Work w;
  const int64_t chunk = std::min<int64_t>(n_out, kChunkRows);
  SG_TRY(mlp_work(m, chunk, false, w));
  for (int64_t s0 = 0; s0 < n_out; s0 += chunk) {
    Walk walk{nullptr, 0, 0, s0, n * q, n, holdout, 1};
    SG_TRY(forward_rows(m, F, nullptr, walk, std::min<int64_t>(chunk, n_out - s0), w, false,
                        y.as<float>() + s0, st));
  }
  const int blocks = (int)std::min<int64_t>((n_out + 255) / 256, 1024);
  SG_TRY(part.reserve((size_t)blocks * 2 * sizeof(double)));
  const Walk vw{nullptr, 0, 0, 0, n * q, n, holdout, 1};
  mlp_val_kernel<<<(unsigned)blocks, 256, 0, st>>>(y.as<float>(), T, vw, n_out, part.as<double>());
  count_launches(1);
  SG_CHECK_LAUNCH();
  std::vector<double> h((size_t)blocks * 2);
  SG_CUDA(cudaMemcpyAsync(h.data(), part.ptr, h.size() * 8, cudaMemcpyDeviceToHost, st));
  SG_TRY(check_err(m, st));
  double se = 0.0, stt = 0.0;
  for (int b = 0; b < blocks; ++b) {
    se += h[(size_t)2 * b];
    stt += h[(size_t)2 * b + 1];
  }
  *mse = se / (double)n_out;
  *target_ms = stt / (double)n_out;
  return Status();
}

}  // namespace saige

using namespace saige;

#define SG_API extern "C" __attribute__((visibility("default")))

namespace {
struct StreamGuard {
  cudaStream_t s = nullptr;
  ~StreamGuard() {
    if (s) cudaStreamDestroy(s);
  }
};
}  // namespace

SG_API int32_t saige_mlp_param_count(void) { return kMlpParams; }

SG_API int32_t saige_mlp_initial_params(uint64_t seed, float* params) {
  if (!params) return fail(SAIGE_EINVAL, "null argument").code;
  std::vector<float> w;
  mlp_initial_weights(seed, w);
  memcpy(params, w.data(), w.size() * sizeof(float));
  return SAIGE_OK;
}

SG_API int32_t saige_mlp_eval(const float* params, const float* features, const float* targets,
                              int64_t n_ex, float* out, float* grad, double* sse, int32_t device) {
  try {
    set_error("");
    if (!params || !features || n_ex <= 0 || ((grad || sse) && !targets))
      return fail(SAIGE_EINVAL, "null argument or empty input").code;
    int dev = 0;
    Status s = pick_device(device, &dev);
    if (!s.ok()) return s.code;
    StreamGuard sg;
    if (cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking) != cudaSuccess)
      return fail(SAIGE_ECUDA, "stream creation failed").code;
    auto body = [&]() -> Status {
      Mlp m;
      SG_TRY(mlp_alloc(m));
      SG_TRY(mlp_set(m, params, sg.s));
      DevBuf F, T, Y;
      SG_TRY(F.reserve((size_t)n_ex * kMlpIn * 4));
      SG_CUDA(cudaMemcpyAsync(F.ptr, features, (size_t)n_ex * kMlpIn * 4, cudaMemcpyHostToDevice,
                              sg.s));
      if (targets) {
        SG_TRY(T.reserve((size_t)n_ex * 4));
        SG_CUDA(cudaMemcpyAsync(T.ptr, targets, (size_t)n_ex * 4, cudaMemcpyHostToDevice, sg.s));
      }
      if (out) {
        SG_TRY(Y.reserve((size_t)n_ex * 4));
        SG_TRY(mlp_forward(m, F.as<float>(), n_ex, Y.as<float>(), sg.s));
        SG_CUDA(cudaMemcpyAsync(out, Y.ptr, (size_t)n_ex * 4, cudaMemcpyDeviceToHost, sg.s));
      }
      if (grad || sse) {
        SG_TRY(mlp_grad(m, F.as<float>(), T.as<float>(), n_ex, sg.s));
        if (grad)
          SG_CUDA(cudaMemcpyAsync(grad, m.grad, (size_t)kMlpParams * 4, cudaMemcpyDeviceToHost,
                                  sg.s));
        if (sse) SG_CUDA(cudaMemcpyAsync(sse, m.loss, sizeof(double), cudaMemcpyDeviceToHost, sg.s));
      }
      SG_CUDA(cudaStreamSynchronize(sg.s));
      return check_err(m, sg.s);
    };
    return body().code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}

SG_API int32_t saige_mlp_train(float* params, const float* features, const float* targets,
                               int64_t n, int32_t q, int32_t steps, float lr, int32_t holdout,
                               double* val_mse_before, double* val_mse_after,
                               double* val_target_ms, int32_t device) {
  try {
    set_error("");
    if (!params || !features || !targets || n <= 0 || q <= 0 || steps < 0 || holdout < 2)
      return fail(SAIGE_EINVAL, "null argument or bad size").code;
    int dev = 0;
    Status s = pick_device(device, &dev);
    if (!s.ok()) return s.code;
    StreamGuard sg;
    if (cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking) != cudaSuccess)
      return fail(SAIGE_ECUDA, "stream creation failed").code;
    auto body = [&]() -> Status {
      Mlp m;
      SG_TRY(mlp_alloc(m));
      SG_TRY(mlp_set(m, params, sg.s));
      const int64_t n_ex = n * q;
      DevBuf F, T;
      SG_TRY(F.reserve((size_t)n_ex * kMlpIn * 4));
      SG_TRY(T.reserve((size_t)n_ex * 4));
      SG_CUDA(cudaMemcpyAsync(F.ptr, features, (size_t)n_ex * kMlpIn * 4, cudaMemcpyHostToDevice,
                              sg.s));
      SG_CUDA(cudaMemcpyAsync(T.ptr, targets, (size_t)n_ex * 4, cudaMemcpyHostToDevice, sg.s));
      double mse = 0.0, tms = 0.0;
      SG_TRY(mlp_validate(m, F.as<float>(), T.as<float>(), n, q, holdout, &mse, &tms, sg.s));
      if (val_mse_before) *val_mse_before = mse;
      SG_TRY(mlp_train(m, F.as<float>(), T.as<float>(), n, q, steps, lr, holdout, sg.s));
      SG_TRY(mlp_validate(m, F.as<float>(), T.as<float>(), n, q, holdout, &mse, &tms, sg.s));
      if (val_mse_after) *val_mse_after = mse;
      if (val_target_ms) *val_target_ms = tms;
      SG_CUDA(cudaMemcpyAsync(params, m.master, (size_t)kMlpParams * 4, cudaMemcpyDeviceToHost,
                              sg.s));
      SG_CUDA(cudaStreamSynchronize(sg.s));
      return Status();
    };
    return body().code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}
