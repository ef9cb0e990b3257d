// Shared plumbing for the sm_100a fit-null library: status codes, error
// capture, device helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
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

// With SAIGE_TIMING=1 in the environment, saige_fit_null_from_bed, the GRM handle
// build and the AI-REML fit print the wall time of each phase (device synchronised
// at each mark) to stderr.
struct PhaseTimer {
  bool on = false;
  const int64_t* launches = nullptr;  // GRM product launches, reported per phase when set
  int64_t l0 = 0;
  std::chrono::steady_clock::time_point t0;
  PhaseTimer() {
    const char* e = getenv("SAIGE_TIMING");
    on = e && e[0] == '1';
    t0 = std::chrono::steady_clock::now();
  }
  void mark(const char* what) {
    if (!on) return;
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    const int64_t l = launches ? *launches : 0;
    fprintf(stderr, "[saige timing] %-10s %8.2f ms  %lld GRM launches\n", what,
            std::chrono::duration<double, std::milli>(t1 - t0).count(), (long long)(l - l0));
    l0 = l;
    t0 = t1;
  }
};

}  // namespace saige
