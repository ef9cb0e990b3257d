// Shared plumbing for the sm_100a fit-null library: status codes, error
// capture, device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/saige_gpu.h"

namespace saige {

void set_error(const std::string& msg);
const char* last_error();

struct Status {
  int32_t code = SAIGE_OK;
  Status() = default;
  Status(int32_t c) : code(c) {}
  bool ok() const { return code == SAIGE_OK; }
};

Status fail(int32_t code, const char* fmt, ...);

// Process-wide count of kernels launched by this library.
void count_launches(int k);
int64_t launches_total();

#define SG_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t _e = (call);                                                           \
    if (_e != cudaSuccess)                                                             \
      return ::saige::fail(SAIGE_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,      \
                           cudaGetErrorString(_e));                                    \
  } while (0)

#define SG_TRY(expr)                   \
  do {                                 \
    ::saige::Status _s = (expr);       \
    if (!_s.ok()) return _s;           \
  } while (0)

#define SG_CHECK_LAUNCH() SG_CUDA(cudaGetLastError())

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Sample padding unit: rows of the packed genotype matrix hold a multiple of
// 512 samples (128 bytes), so every row starts 128-byte aligned.
constexpr int64_t kSamplePad = 512;
// Marker padding unit: a multiple of the 128-row tensor-core tile.
constexpr int64_t kMarkerPad = 128;

// Device-side warp reductions.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace saige
