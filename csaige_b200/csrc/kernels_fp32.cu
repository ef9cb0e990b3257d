// FP32 GRM product on CUDA cores: the saige-rs arithmetic of
// OnTheFlyGrm::mat_vec (saige-core/src/glmm/pcg.rs:128-180) — z rounded to
// f32 per marker and code exactly as OnTheFlyGrm::new (pcg.rs:101-122), v
// rounded to f32, f32 products and sums — read straight from the 2-bit rows.
//
// Decode: each nibble of a packed word holds two samples' codes (the device
// word layout pairs samples (k, k+4) and (k+4, k+8)); the nibble indexes a
// per-marker table of 16 float2 entries (z(code_lo), z(code_hi)) held in
// shared memory, so one 64-bit shared load plus one packed f32x2 FMA covers
// two samples.  The 16
// entries span all 32 banks, so a warp's lookups never conflict.
//   pass A  u_m  = sum_i z_mi v_i        (CTA = 16 markers x all samples)
//   pass B  y_i  = sum_m z_mi u_m        (CTA = 4096 samples x a marker split)
// Pass B writes per-split partial sums, summed in a fixed order by the finish
// kernel, so results are run-to-run deterministic.
#include "common.cuh"
#include "kernels.cuh"

namespace saige {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMarkersA = 16;   // markers per CTA in pass A
constexpr int kChunkB = 128;    // markers per table chunk in pass B
constexpr int kWindowWords = kThreads;  // pass B: one 32-bit code word per thread

__device__ __forceinline__ float zsel(const float4& z, int c) {
  return c == 0 ? z.x : (c == 1 ? z.y : (c == 2 ? z.z : z.w));
}

__global__ void __launch_bounds__(kThreads)
    fp32_zt_kernel(const uint32_t* __restrict__ geno, int64_t wpr, const float4* __restrict__ zlut,
                   const float* __restrict__ v32, float* __restrict__ u) {
  __shared__ float2 tab[kMarkersA][16];
  __shared__ float part[kWarps][kMarkersA];
  const int64_t m0 = (int64_t)blockIdx.x * kMarkersA;
  for (int e = threadIdx.x; e < kMarkersA * 16; e += kThreads) {
    const int mb = e >> 4, nib = e & 15;
    const float4 z = zlut[m0 + mb];
    tab[mb][nib] = make_float2(zsel(z, nib & 3), zsel(z, nib >> 2));
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float2 acc[kMarkersA];
#pragma unroll
  for (int mb = 0; mb < kMarkersA; ++mb) acc[mb] = make_float2(0.f, 0.f);
  const int64_t n_steps = wpr / 32;
  const uint32_t* rows = geno + m0 * wpr;
  for (int64_t s = warp; s < n_steps; s += kWarps) {
    const int64_t wo = s * 32 + lane;
    const float4* vp = reinterpret_cast<const float4*>(v32 + wo * 16);
    // nibble k of a device-layout word holds samples (k, k+4) for k < 4 and
    // (k+4, k+8) for k >= 4
    const float4 f0 = __ldg(vp), f1 = __ldg(vp + 1), f2 = __ldg(vp + 2), f3 = __ldg(vp + 3);
    const float2 vv[8] = {make_float2(f0.x, f1.x), make_float2(f0.y, f1.y), make_float2(f0.z, f1.z),
                          make_float2(f0.w, f1.w), make_float2(f2.x, f3.x), make_float2(f2.y, f3.y),
                          make_float2(f2.z, f3.z), make_float2(f2.w, f3.w)};
    uint32_t w[kMarkersA];
#pragma unroll
    for (int mb = 0; mb < kMarkersA; ++mb) w[mb] = __ldg(rows + mb * wpr + wo);
#pragma unroll
    for (int mb = 0; mb < kMarkersA; ++mb) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float2 t = tab[mb][(w[mb] >> (4 * k)) & 15u];
        acc[mb] = __ffma2_rn(t, vv[k], acc[mb]);
      }
    }
  }
#pragma unroll
  for (int mb = 0; mb < kMarkersA; ++mb) {
    float t = warp_sum(acc[mb].x + acc[mb].y);
    if (lane == 0) part[warp][mb] = t;
  }
  __syncthreads();
  if (threadIdx.x < kMarkersA) {
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < kWarps; ++q) s += part[q][threadIdx.x];
    u[m0 + threadIdx.x] = s;
  }
}

__global__ void __launch_bounds__(kThreads)
    fp32_z_kernel(const uint32_t* __restrict__ geno, int64_t wpr, const float4* __restrict__ zlut,
                  int64_t m_pad, const float* __restrict__ u, float* __restrict__ ypart,
                  int64_t n_pad, int64_t per_split) {
  __shared__ float2 tab[2][kChunkB][16];
  const int64_t ms = (int64_t)blockIdx.y * per_split;
  int64_t me = ms + per_split;
  if (me > m_pad) me = m_pad;
  const int64_t wo = (int64_t)blockIdx.x * kWindowWords + threadIdx.x;
  const bool active = wo < wpr;
  float2 acc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc[k] = make_float2(0.f, 0.f);
  int buf = 0;
  for (int64_t c0 = ms; c0 < me; c0 += kChunkB) {
    for (int e = threadIdx.x; e < kChunkB * 16; e += kThreads) {
      const int mb = e >> 4, nib = e & 15;
      const int64_t m = c0 + mb;
      float2 t = make_float2(0.f, 0.f);
      if (m < me) {
        const float4 z = zlut[m];
        const float um = u[m];
        t = make_float2(zsel(z, nib & 3) * um, zsel(z, nib >> 2) * um);
      }
      tab[buf][mb][nib] = t;
    }
    __syncthreads();
    if (active) {
      const int cnt = (int)((me - c0) < kChunkB ? (me - c0) : kChunkB);
      const uint32_t* p = geno + c0 * wpr + wo;
      int mb = 0;
      for (; mb + 4 <= cnt; mb += 4) {
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = __ldg(p + (int64_t)(mb + q) * wpr);
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int k = 0; k < 8; ++k) acc[k] = __fadd2_rn(acc[k], tab[buf][mb + q][(w[q] >> (4 * k)) & 15u]);
      }
      for (; mb < cnt; ++mb) {
        const uint32_t w = __ldg(p + (int64_t)mb * wpr);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = __fadd2_rn(acc[k], tab[buf][mb][(w >> (4 * k)) & 15u]);
      }
    }
    buf ^= 1;
  }
  if (active) {
    float4* o = reinterpret_cast<float4*>(ypart + (int64_t)blockIdx.y * n_pad + wo * 16);
    o[0] = make_float4(acc[0].x, acc[1].x, acc[2].x, acc[3].x);
    o[1] = make_float4(acc[0].y, acc[1].y, acc[2].y, acc[3].y);
    o[2] = make_float4(acc[4].x, acc[5].x, acc[6].x, acc[7].x);
    o[3] = make_float4(acc[4].y, acc[5].y, acc[6].y, acc[7].y);
  }
}

__global__ void fp32_finish_kernel(const float* __restrict__ ypart, int n_splits, int64_t n_pad,
                                   int64_t n, float scale, double* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int q = 0; q < n_splits; ++q) s += ypart[(int64_t)q * n_pad + i];
  out[i] = (double)(s * scale);
}

__global__ void to_f32_kernel(const double* __restrict__ v, int64_t n, int64_t n_pad,
                              float* __restrict__ v32) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_pad) v32[i] = i < n ? (float)v[i] : 0.f;
}

}  // namespace

int fp32_z_splits(int64_t n_pad, int64_t m_pad) {
  const int64_t windows = ceil_div(n_pad / 16, kWindowWords);
  int64_t want = ceil_div(148 * 6, windows);
  const int64_t max_splits = ceil_div(m_pad, kChunkB);
  if (want > max_splits) want = max_splits;
  if (want < 1) want = 1;
  return (int)want;
}

cudaError_t launch_fp32_zt(const uint32_t* geno, int64_t wpr, const float4* zlut, int64_t m_pad,
                           const float* v32, float* u, cudaStream_t st) {
  fp32_zt_kernel<<<(unsigned)(m_pad / kMarkersA), kThreads, 0, st>>>(geno, wpr, zlut, v32, u);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fp32_z(const uint32_t* geno, int64_t wpr, const float4* zlut, int64_t m_pad,
                          const float* u, float* ypart, int n_splits, cudaStream_t st) {
  const int64_t windows = ceil_div(wpr, kWindowWords);
  const int64_t per_split = round_up(ceil_div(m_pad, n_splits), 4);
  dim3 grid((unsigned)windows, (unsigned)n_splits);
  fp32_z_kernel<<<grid, kThreads, 0, st>>>(geno, wpr, zlut, m_pad, u, ypart, wpr * 16, per_split);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_fp32_finish(const float* ypart, int n_splits, int64_t n_pad, int64_t n,
                               float scale, double* out, cudaStream_t st) {
  fp32_finish_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(ypart, n_splits, n_pad, n, scale,
                                                                 out);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_to_f32(const double* v, int64_t n, int64_t n_pad, float* v32, cudaStream_t st) {
  to_f32_kernel<<<(unsigned)ceil_div(n_pad, 256), 256, 0, st>>>(v, n, n_pad, v32);
  count_launches(1);
  return cudaGetLastError();
}

}  // namespace saige
