// The MLP of the learned warm start: fused forward (inference) and fused
// forward + backward (training) kernels on the CUDA cores with BF16 weights and FP32
// arithmetic, an Adam kernel, and the training loop captured as one CUDA graph.
//
// Examples are (sample, column) pairs e = c * n + i with 8 features F[e*8 .. e*8+8]
// and a target T[e].  Layers: h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2),
// h3 = tanh(W3 h2 + b3), y = w4 . h3 + b4 (64 units each).  The forward passes use
// the BF16 copy of the weights; the gradient is taken with respect to the FP32 master
// weights through that rounding (straight through).  Per-block gradient partials are
// summed in a fixed order, so training is deterministic.
#include <cuda_bf16.h>

#include <string.h>

#include <cmath>
#include <mutex>
#include <set>
#include <vector>

#include "mlp.cuh"

namespace saige {
namespace {

constexpr int kFwdThreads = 256;
constexpr int kTrainThreads = 128;
constexpr int kTrainBlocksMax = 256;
constexpr int H = kMlpH;
constexpr int IN = kMlpIn;

__device__ __forceinline__ float bf16_to_f32(uint16_t b) {
  return __uint_as_float((uint32_t)b << 16);
}

// Weights in shared memory, each matrix transposed to [in][out] so that one float4
// load serves four outputs of one input.
struct SmemW {
  float* w1t;  // [IN][H]
  float* b1;
  float* w2t;  // [H][H]
  float* b2;
  float* w3t;  // [H][H]
  float* b3;
  float* w4;
  float* b4;
};
constexpr int kSmemWFloats = IN * H + H + H * H + H + H * H + H + H + 4;

__device__ SmemW carve_w(float* s) {
  SmemW w;
  w.w1t = s;
  w.b1 = w.w1t + IN * H;
  w.w2t = w.b1 + H;
  w.b2 = w.w2t + H * H;
  w.w3t = w.b2 + H;
  w.b3 = w.w3t + H * H;
  w.w4 = w.b3 + H;
  w.b4 = w.w4 + H;
  return w;
}

__device__ void load_w(const uint16_t* __restrict__ wbf, SmemW w) {
  for (int t = threadIdx.x; t < H * IN; t += blockDim.x) {
    const int j = t / IN, k = t % IN;
    w.w1t[k * H + j] = bf16_to_f32(wbf[kMlpW1 + t]);
  }
  for (int t = threadIdx.x; t < H * H; t += blockDim.x) {
    const int j = t / H, k = t % H;
    w.w2t[k * H + j] = bf16_to_f32(wbf[kMlpW2 + t]);
    w.w3t[k * H + j] = bf16_to_f32(wbf[kMlpW3 + t]);
  }
  for (int t = threadIdx.x; t < H; t += blockDim.x) {
    w.b1[t] = bf16_to_f32(wbf[kMlpB1 + t]);
    w.b2[t] = bf16_to_f32(wbf[kMlpB2 + t]);
    w.b3[t] = bf16_to_f32(wbf[kMlpB3 + t]);
    w.w4[t] = bf16_to_f32(wbf[kMlpW4 + t]);
  }
  if (threadIdx.x == 0) w.b4[0] = bf16_to_f32(wbf[kMlpB4]);
}

// out[j][t] = tanh(b[j] + sum_k wt[k][j] in[k][t]) for j < H; in/out: [units][T] floats.
template <int K, int T>
__device__ __forceinline__ void dense_tanh(const float* __restrict__ wt, const float* __restrict__ b,
                                           const float* in, float* out, int t) {
  for (int jb = 0; jb < H; jb += 8) {
    float s[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) s[i] = b[jb + i];
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
      const float a = in[k * T + t];
      const float4 w0 = *reinterpret_cast<const float4*>(wt + k * H + jb);
      const float4 w1 = *reinterpret_cast<const float4*>(wt + k * H + jb + 4);
      s[0] += w0.x * a; s[1] += w0.y * a; s[2] += w0.z * a; s[3] += w0.w * a;
      s[4] += w1.x * a; s[5] += w1.y * a; s[6] += w1.z * a; s[7] += w1.w * a;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) out[(jb + i) * T + t] = tanhf(s[i]);
  }
}

template <int T>
__device__ __forceinline__ float forward_one(SmemW w, float* a0, float* a1, float* a2, float* a3,
                                             int t) {
  dense_tanh<IN, T>(w.w1t, w.b1, a0, a1, t);
  dense_tanh<H, T>(w.w2t, w.b2, a1, a2, t);
  dense_tanh<H, T>(w.w3t, w.b3, a2, a3, t);
  float y = w.b4[0];
#pragma unroll 8
  for (int k = 0; k < H; ++k) y += w.w4[k] * a3[k * T + t];
  return y;
}

// Logical example j: e = j when holdout == 0; otherwise the held-out examples only,
// j = c * nh + h with nh = ceil(n / holdout), e = c * n + h * holdout.
__global__ void __launch_bounds__(kFwdThreads)
    mlp_forward_kernel(const uint16_t* __restrict__ wbf, const float* __restrict__ F, int64_t n_ex,
                       int64_t n, int holdout, float* __restrict__ out) {
  extern __shared__ __align__(16) float smem[];
  const SmemW w = carve_w(smem);
  float* act = smem + kSmemWFloats;  // a0 [IN][T], a1/a2 ping-pong [H][T]
  float* a0 = act;
  float* a1 = a0 + IN * kFwdThreads;
  float* a2 = a1 + H * kFwdThreads;
  load_w(wbf, w);
  __syncthreads();
  const int t = threadIdx.x;
  const int64_t nh = holdout > 0 ? (n + holdout - 1) / holdout : 0;
  for (int64_t base = (int64_t)blockIdx.x * kFwdThreads; base < n_ex;
       base += (int64_t)gridDim.x * kFwdThreads) {
    const int64_t j = base + t;
    if (j < n_ex) {
      const int64_t e = holdout > 0 ? (j / nh) * n + (j % nh) * holdout : j;
      const float4 f0 = *reinterpret_cast<const float4*>(F + e * IN);
      const float4 f1 = *reinterpret_cast<const float4*>(F + e * IN + 4);
      const float f[8] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w};
#pragma unroll
      for (int k = 0; k < IN; ++k) a0[k * kFwdThreads + t] = f[k];
      // a1 -> a2 -> a1 reuse: the third layer writes into a1
      dense_tanh<IN, kFwdThreads>(w.w1t, w.b1, a0, a1, t);
      dense_tanh<H, kFwdThreads>(w.w2t, w.b2, a1, a2, t);
      dense_tanh<H, kFwdThreads>(w.w3t, w.b3, a2, a1, t);
      float y = w.b4[0];
#pragma unroll 8
      for (int k = 0; k < H; ++k) y += w.w4[k] * a1[k * kFwdThreads + t];
      out[j] = y;
    }
  }
}

// dW[j][k] (j < J, k < K) partial over the block's T examples: g [J][T], a [K][T];
// thread tid owns a 4 x 8 block of entries when J * K / 32 >= T (the H x H layers)
// or one row slice otherwise.
template <int J, int K, int T>
__device__ __forceinline__ void outer_sum(const float* g, const float* a, float* dst, int tid) {
  constexpr int kBlocks = (J / 4) * (K / 8);
  for (int blk = tid; blk < kBlocks; blk += T) {
    const int j0 = (blk / (K / 8)) * 4, k0 = (blk % (K / 8)) * 8;
    float acc[4][8];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;
    for (int e = 0; e < T; ++e) {
      float gv[4], av[8];
#pragma unroll
      for (int r = 0; r < 4; ++r) gv[r] = g[(j0 + r) * T + e];
#pragma unroll
      for (int c = 0; c < 8; ++c) av[c] = a[(k0 + c) * T + e];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] += gv[r] * av[c];
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c) dst[(j0 + r) * K + k0 + c] = acc[r][c];
  }
}

// One block = kTrainThreads examples.  Writes its gradient partial (kMlpParams floats)
// to part[blockIdx.x] and its summed squared error to lpart[blockIdx.x].
// Example slot s of the pass: e = idx ? idx[s] : (stride ? (s0 + s) * stride % n_ex : s);
// slots past n_slots, and examples whose sample index (e % n) % holdout == 0 when
// holdout > 0, carry no weight.
__global__ void __launch_bounds__(kTrainThreads)
    mlp_grad_kernel(const uint16_t* __restrict__ wbf, const float* __restrict__ F,
                    const float* __restrict__ Tg, const int64_t* __restrict__ idx, int64_t n_ex,
                    int64_t n_slots, const int* __restrict__ step, int64_t batch, int64_t stride,
                    int64_t n, int holdout, float scale, float* __restrict__ part,
                    double* __restrict__ lpart) {
  extern __shared__ __align__(16) float smem[];
  const SmemW w = carve_w(smem);
  constexpr int T = kTrainThreads;
  float* a0 = smem + kSmemWFloats;  // [IN][T]
  float* a1 = a0 + IN * T;          // [H][T], later g1
  float* a2 = a1 + H * T;           // later g2
  float* a3 = a2 + H * T;           // later g3
  __shared__ float gy[T];
  __shared__ double red[T / 32];
  load_w(wbf, w);
  const int t = threadIdx.x;
  const int64_t s0 = step ? (int64_t)(*step) * batch : 0;
  const int64_t slot = (int64_t)blockIdx.x * T + t;
  int64_t e = -1;
  if (slot < n_slots) {
    if (idx) e = idx[slot];
    else if (stride) e = (int64_t)(((unsigned long long)(s0 + slot) * (unsigned long long)stride) %
                                   (unsigned long long)n_ex);
    else e = slot;
  }
  bool use = e >= 0 && e < n_ex;
  if (use && holdout > 0 && ((e % n) % holdout) == 0) use = false;
  float f[IN] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float target = 0.f;
  if (use) {
    const float4 f0 = *reinterpret_cast<const float4*>(F + e * IN);
    const float4 f1 = *reinterpret_cast<const float4*>(F + e * IN + 4);
    f[0] = f0.x; f[1] = f0.y; f[2] = f0.z; f[3] = f0.w;
    f[4] = f1.x; f[5] = f1.y; f[6] = f1.z; f[7] = f1.w;
    target = Tg[e];
  }
#pragma unroll
  for (int k = 0; k < IN; ++k) a0[k * T + t] = f[k];
  __syncthreads();
  const float y = forward_one<T>(w, a0, a1, a2, a3, t);
  const float err = use ? y - target : 0.f;
  const float g_y = 2.f * err * scale;  // d/dy of scale * sum err^2
  gy[t] = g_y;
  // g3 = g_y w4 (1 - h3^2), in place of h3 after dw4 is formed below
  float* P = part + (int64_t)blockIdx.x * kMlpParams;
  __syncthreads();
  // dw4[k] = sum_t g_y h3[k][t]; db4 = sum_t g_y
  for (int k = t; k < H; k += T) {
    float s = 0.f;
    for (int e2 = 0; e2 < T; ++e2) s += gy[e2] * a3[k * T + e2];
    P[kMlpW4 + k] = s;
  }
  if (t == 0) {
    float s = 0.f;
    for (int e2 = 0; e2 < T; ++e2) s += gy[e2];
    P[kMlpB4] = s;
  }
  __syncthreads();
#pragma unroll 8
  for (int k = 0; k < H; ++k) {
    const float h = a3[k * T + t];
    a3[k * T + t] = g_y * w.w4[k] * (1.f - h * h);
  }
  __syncthreads();
  // layer 3: dW3 = g3 h2', db3 = sum g3; g2 = (W3' g3)(1 - h2^2)
  outer_sum<H, H, T>(a3, a2, P + kMlpW3, t);
  for (int j = t; j < H; j += T) {
    float s = 0.f;
    for (int e2 = 0; e2 < T; ++e2) s += a3[j * T + e2];
    P[kMlpB3 + j] = s;
  }
  __syncthreads();
  for (int kb = 0; kb < H; kb += 8) {
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
      const float g = a3[j * T + t];
      // W3[j][k] = w3t[k][j]
#pragma unroll
      for (int i = 0; i < 8; ++i) s[i] += w.w3t[(kb + i) * H + j] * g;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float h = a2[(kb + i) * T + t];
      a2[(kb + i) * T + t] = s[i] * (1.f - h * h);
    }
  }
  __syncthreads();
  // layer 2
  outer_sum<H, H, T>(a2, a1, P + kMlpW2, t);
  for (int j = t; j < H; j += T) {
    float s = 0.f;
    for (int e2 = 0; e2 < T; ++e2) s += a2[j * T + e2];
    P[kMlpB2 + j] = s;
  }
  __syncthreads();
  for (int kb = 0; kb < H; kb += 8) {
    float s[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll 4
    for (int j = 0; j < H; ++j) {
      const float g = a2[j * T + t];
#pragma unroll
      for (int i = 0; i < 8; ++i) s[i] += w.w2t[(kb + i) * H + j] * g;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float h = a1[(kb + i) * T + t];
      a1[(kb + i) * T + t] = s[i] * (1.f - h * h);
    }
  }
  __syncthreads();
  // layer 1: dW1 = g1 x', db1 = sum g1
  outer_sum<H, IN, T>(a1, a0, P + kMlpW1, t);
  for (int j = t; j < H; j += T) {
    float s = 0.f;
    for (int e2 = 0; e2 < T; ++e2) s += a1[j * T + e2];
    P[kMlpB1 + j] = s;
  }
  // squared error of the block
  double se = use ? (double)err * (double)err : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
  if ((t & 31) == 0) red[t >> 5] = se;
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int i = 0; i < T / 32; ++i) s += red[i];
    lpart[blockIdx.x] = s;
  }
}

// grad[p] = sum over blocks (in order) of part[b][p]; loss[0] = sum of lpart.
__global__ void mlp_sum_kernel(const float* __restrict__ part, const double* __restrict__ lpart,
                               int nblocks, float* __restrict__ grad, double* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) {
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += part[(int64_t)b * kMlpParams + p];
    grad[p] = s;
  }
  if (p == 0) {
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += lpart[b];
    loss[0] = s;
  }
}

// Adam (Kingma and Ba, 2015) on the summed block partials; then the BF16 copy.
__global__ void mlp_adam_kernel(const float* __restrict__ part, int nblocks, float* __restrict__ w,
                                uint16_t* __restrict__ wbf, float* __restrict__ m1,
                                float* __restrict__ m2, int* __restrict__ step, float lr) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = *step + 1;
  if (p < kMlpParams) {
    float g = 0.f;
    for (int b = 0; b < nblocks; ++b) g += part[(int64_t)b * kMlpParams + p];
    const float b1 = 0.9f, b2 = 0.999f;
    const float mm = b1 * m1[p] + (1.f - b1) * g;
    const float vv = b2 * m2[p] + (1.f - b2) * g * g;
    m1[p] = mm;
    m2[p] = vv;
    const float mh = mm / (1.f - powf(b1, (float)s));
    const float vh = vv / (1.f - powf(b2, (float)s));
    const float nw = w[p] - lr * mh / (sqrtf(vh) + 1e-8f);
    w[p] = nw;
    wbf[p] = __bfloat16_as_ushort(__float2bfloat16_rn(nw));
  }
  // every thread has read *step above; the grid-wide increment happens in the next launch
}

__global__ void mlp_step_kernel(int* step) { *step += 1; }

__global__ void mlp_to_bf16_kernel(const float* __restrict__ w, uint16_t* __restrict__ wbf) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kMlpParams) wbf[p] = __bfloat16_as_ushort(__float2bfloat16_rn(w[p]));
}

// Held-out squared error and squared target: y[j] is the output of held-out example j
// (see mlp_forward_kernel), T the targets of all examples.
__global__ void mlp_val_kernel(const float* __restrict__ y, const float* __restrict__ Tg,
                               int64_t n_out, int64_t n, int holdout, double* __restrict__ part) {
  __shared__ double sh[2][8];
  const int64_t nh = (n + holdout - 1) / holdout;
  double se = 0.0, st = 0.0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_out;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = (j / nh) * n + (j % nh) * holdout;
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

constexpr size_t kFwdSmem = (size_t)(kSmemWFloats + IN * kFwdThreads + 2 * H * kFwdThreads) * 4;
constexpr size_t kTrainSmem = (size_t)(kSmemWFloats + IN * kTrainThreads + 3 * H * kTrainThreads) * 4;

// The dynamic shared-memory limits are a per-device attribute: set once per device.
cudaError_t set_smem_attrs() {
  static std::mutex mu;
  static std::set<int> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count(dev)) return cudaSuccess;
  e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kFwdSmem);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kTrainSmem);
  if (e == cudaSuccess) done.insert(dev);
  return e;
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

Status mlp_partials(Mlp& m, int blocks) {
  if (m.part_blocks >= blocks) return Status();
  SG_TRY(m.part.reserve((size_t)blocks * kMlpParams * sizeof(float)));
  SG_TRY(m.lpart.reserve((size_t)blocks * sizeof(double)));
  m.part_blocks = blocks;
  return Status();
}

constexpr int kGraphSteps = 25;

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
  SG_TRY(m.mem.reserve(nf * 4 * 4 + nf * 2 + 64 + 16));
  char* b = m.mem.as<char>();
  m.master = reinterpret_cast<float*>(b);
  m.grad = m.master + nf;
  m.m1 = m.grad + nf;
  m.m2 = m.m1 + nf;
  m.loss = reinterpret_cast<double*>(m.m2 + nf);
  m.step = reinterpret_cast<int*>(m.loss + 2);
  m.wbf = reinterpret_cast<uint16_t*>(m.step + 4);
  return Status();
}

Status mlp_set(Mlp& m, const float* host_w, cudaStream_t st) {
  const size_t nf = (size_t)kMlpParams;
  SG_CUDA(cudaMemcpyAsync(m.master, host_w, nf * 4, cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemsetAsync(m.m1, 0, nf * 4 * 2, st));
  SG_CUDA(cudaMemsetAsync(m.step, 0, 4 * sizeof(int), st));
  mlp_to_bf16_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(m.master, m.wbf);
  count_launches(1);
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

Status mlp_forward(const Mlp& m, const float* F, int64_t n_ex, float* out, cudaStream_t st) {
  if (n_ex <= 0) return Status();
  SG_CUDA(set_smem_attrs());
  const int64_t blocks = std::min<int64_t>(ceil_div(n_ex, kFwdThreads), 148 * 8);
  mlp_forward_kernel<<<(unsigned)blocks, kFwdThreads, kFwdSmem, st>>>(m.wbf, F, n_ex, n_ex, 0, out);
  count_launches(1);
  SG_CHECK_LAUNCH();
  return Status();
}

Status mlp_grad(Mlp& m, const float* F, const float* T, const int64_t* idx, int64_t n_ex,
                cudaStream_t st) {
  SG_CUDA(set_smem_attrs());
  const int blocks = (int)ceil_div(std::max<int64_t>(n_ex, 1), kTrainThreads);
  DevBuf part, lpart;
  SG_TRY(part.reserve((size_t)blocks * kMlpParams * sizeof(float)));
  SG_TRY(lpart.reserve((size_t)blocks * sizeof(double)));
  const float scale = 1.0f / (float)std::max<int64_t>(n_ex, 1);
  mlp_grad_kernel<<<(unsigned)blocks, kTrainThreads, kTrainSmem, st>>>(
      m.wbf, F, T, idx, n_ex, n_ex, nullptr, 0, 0, std::max<int64_t>(n_ex, 1), 0, scale,
      part.as<float>(), lpart.as<double>());
  mlp_sum_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(part.as<float>(), lpart.as<double>(),
                                                          blocks, m.grad, m.loss);
  count_launches(2);
  SG_CHECK_LAUNCH();
  SG_CUDA(cudaStreamSynchronize(st));
  return Status();
}

Status mlp_train(Mlp& m, const float* F, const float* T, int64_t n, int q, int steps, int batch,
                 float lr, int holdout, cudaStream_t st) {
  if (steps <= 0) return Status();
  SG_CUDA(set_smem_attrs());
  const int64_t n_ex = n * q;
  const int blocks = std::min<int>(kTrainBlocksMax, (int)ceil_div(batch, kTrainThreads));
  const int64_t slots = (int64_t)blocks * kTrainThreads;
  const int per = std::min(steps, kGraphSteps);
  const bool same = m.graph && m.graph_key[0] == F && m.graph_key[1] == T && m.graph_n == n &&
                    m.graph_q == q && m.graph_batch == batch && m.graph_holdout == holdout &&
                    m.graph_lr == lr && m.graph_steps == per;
  if (!same) {
    if (m.graph) {
      cudaGraphExecDestroy(m.graph);
      m.graph = nullptr;
    }
    SG_TRY(mlp_partials(m, blocks));
    const int64_t stride = batch_stride(n_ex);
    const float scale = 1.0f / (float)slots;
    // the step loop as one graph: grad pass, Adam, step counter
    cudaGraph_t graph = nullptr;
    SG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < per; ++s) {
      mlp_grad_kernel<<<(unsigned)blocks, kTrainThreads, kTrainSmem, st>>>(
          m.wbf, F, T, nullptr, n_ex, slots, m.step, slots, stride, n, holdout, scale,
          m.part.as<float>(), m.lpart.as<double>());
      mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, st>>>(m.part.as<float>(), blocks,
                                                               m.master, m.wbf, m.m1, m.m2, m.step,
                                                               lr);
      mlp_step_kernel<<<1, 1, 0, st>>>(m.step);
    }
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
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
    m.graph_batch = batch;
    m.graph_holdout = holdout;
    m.graph_lr = lr;
    m.graph_steps = per;
  }
  const int launches = (int)ceil_div(steps, per);
  for (int l = 0; l < launches; ++l) SG_CUDA(cudaGraphLaunch(m.graph, st));
  count_launches(3 * per * launches);
  m.trained_steps += (int64_t)per * launches;
  return Status();
}

Status mlp_validate(Mlp& m, const float* F, const float* T, int64_t n, int q, int holdout,
                    double* mse, double* target_ms, cudaStream_t st) {
  const int64_t nh = (n + holdout - 1) / holdout, n_out = nh * q;
  DevBuf y, part;
  SG_TRY(y.reserve((size_t)n_out * sizeof(float)));
  const int blocks = (int)std::min<int64_t>(ceil_div(n_out, 256), 1024);
  SG_TRY(part.reserve((size_t)blocks * 2 * sizeof(double)));
  SG_CUDA(set_smem_attrs());
  const int64_t fb = std::min<int64_t>(ceil_div(n_out, kFwdThreads), 148 * 8);
  mlp_forward_kernel<<<(unsigned)fb, kFwdThreads, kFwdSmem, st>>>(m.wbf, F, n_out, n, holdout,
                                                                 y.as<float>());
  mlp_val_kernel<<<(unsigned)blocks, 256, 0, st>>>(y.as<float>(), T, n_out, n, holdout,
                                                   part.as<double>());
  count_launches(2);
  SG_CHECK_LAUNCH();
  std::vector<double> h((size_t)blocks * 2);
  SG_CUDA(cudaMemcpyAsync(h.data(), part.ptr, h.size() * 8, cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  double se = 0.0, stt = 0.0;
  for (int b = 0; b < blocks; ++b) {
    se += h[(size_t)2 * b];
    stt += h[(size_t)2 * b + 1];
  }
  *mse = n_out ? se / (double)n_out : 0.0;
  *target_ms = n_out ? stt / (double)n_out : 0.0;
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
      SG_CUDA(cudaMemcpyAsync(F.ptr, features, (size_t)n_ex * kMlpIn * 4, cudaMemcpyHostToDevice, sg.s));
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
        SG_TRY(mlp_grad(m, F.as<float>(), T.as<float>(), nullptr, n_ex, sg.s));
        if (grad)
          SG_CUDA(cudaMemcpyAsync(grad, m.grad, (size_t)kMlpParams * 4, cudaMemcpyDeviceToHost, sg.s));
        if (sse) SG_CUDA(cudaMemcpyAsync(sse, m.loss, sizeof(double), cudaMemcpyDeviceToHost, sg.s));
      }
      SG_CUDA(cudaStreamSynchronize(sg.s));
      return Status();
    };
    return body().code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}

SG_API int32_t saige_mlp_train(float* params, const float* features, const float* targets,
                               int64_t n, int32_t q, int32_t steps, int32_t batch, float lr,
                               int32_t holdout, double* val_mse_before, double* val_mse_after,
                               double* val_target_ms, int32_t device) {
  try {
    set_error("");
    if (!params || !features || !targets || n <= 0 || q <= 0 || steps < 0 || batch <= 0 ||
        holdout < 2)
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
      SG_CUDA(cudaMemcpyAsync(F.ptr, features, (size_t)n_ex * kMlpIn * 4, cudaMemcpyHostToDevice, sg.s));
      SG_CUDA(cudaMemcpyAsync(T.ptr, targets, (size_t)n_ex * 4, cudaMemcpyHostToDevice, sg.s));
      double mse = 0.0, tms = 0.0;
      SG_TRY(mlp_validate(m, F.as<float>(), T.as<float>(), n, q, holdout, &mse, &tms, sg.s));
      if (val_mse_before) *val_mse_before = mse;
      SG_TRY(mlp_train(m, F.as<float>(), T.as<float>(), n, q, steps, batch, lr, holdout, sg.s));
      SG_TRY(mlp_validate(m, F.as<float>(), T.as<float>(), n, q, holdout, &mse, &tms, sg.s));
      if (val_mse_after) *val_mse_after = mse;
      if (val_target_ms) *val_target_ms = tms;
      SG_CUDA(cudaMemcpyAsync(params, m.master, (size_t)kMlpParams * 4, cudaMemcpyDeviceToHost, sg.s));
      SG_CUDA(cudaStreamSynchronize(sg.s));
      return Status();
    };
    return body().code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}
