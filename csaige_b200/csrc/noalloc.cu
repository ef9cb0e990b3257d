// GRM product K·v in FP32 arithmetic that allocates no device memory.
//
// saige_grm_matvec_dev grows per-handle workspaces with cudaMalloc on first use
// (and whenever a larger request arrives).  Some callers cannot let a library do
// that: an application that hands almost all of HBM to its own memory pool at
// start-up (a serving process or a framework's caching allocator), where a stray
// cudaMalloc fails or fragments the pool, and a caller on a latency-critical path,
// where cudaMalloc/cudaFree may synchronise the device.  This file gives them
// saige_grm_matvec_dev_noalloc: the same FP32 kernels, with their scratch (the
// f32 copy of v, u = Zᵀv, and the per-split partial sums of Z·u) in one
// fixed-size array compiled into the library.
//
// The array is a file-scope __device__ variable, so every GPU that loads the
// library holds kNoAllocScratchBytes of it until the process exits.  Host code
// may not use the array's name as a device address (on the host it names a
// stand-in object), so the first call on each device looks its address up with
// cudaGetSymbolAddress, with that device current, and later calls reuse it.
// All calls on a device share the one array: calls whose work overlaps on the
// GPU (different streams, or host threads enqueueing at the same time without
// ordering their streams) race on it.  Every element a call reads is written
// earlier in the same call, so nothing carries over between calls.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "engine.cuh"
#include "kernels.cuh"

namespace saige {
namespace {

// 32 MiB.  A handle needs align256(4 n_pad) + align256(4 m_pad) + 4 n_splits n_pad
// bytes of it (noalloc_bytes): the f32 copy of v, u = Z'v and the per-split partial
// sums of Z u, with n_pad = n rounded up to 512, m_pad = m rounded up to 128 and
// n_splits from fp32_z_splits (fewer splits as n grows).  At 150,000 markers that
// admits up to about 2.7 million samples; saige_grm_noalloc_scratch_bytes reports the
// figure of a given handle.
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
struct ScratchAddr {
  CUcontext ctx = nullptr;  // the context the address belongs to
  void* addr = nullptr;
};
ScratchAddr g_scratch_addr[kMaxDevices];

// Device address of g_noalloc_scratch on `device` (current), looked up on the first
// call in each context: a device reset or a new primary context reloads the module,
// and the array may then live elsewhere.
Status scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices)
    return fail(SAIGE_EINVAL, "device %d out of range for the static scratch table", device);
  // the driver's cuCtxGetCurrent through the runtime, so that the library does not
  // link libcuda (it must load on machines without a GPU driver)
  static CUresult (*ctx_get_current)(CUcontext*) = nullptr;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      (void)cudaGetLastError();
      return fail(SAIGE_ECUDA, "cuCtxGetCurrent is not available from the driver");
    }
    ctx_get_current = reinterpret_cast<CUresult (*)(CUcontext*)>(fn);
  }
  CUcontext ctx = nullptr;
  if (ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
    return fail(SAIGE_ECUDA, "no current CUDA context on device %d", device);
  ScratchAddr& e = g_scratch_addr[device];
  if (!e.addr || e.ctx != ctx) {
    void* p = nullptr;
    SG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return fail(SAIGE_ECUDA, "cudaGetSymbolAddress returned a null address");
    e.addr = p;
    e.ctx = ctx;
  }
  *out = e.addr;
  return Status();
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t noalloc_bytes(const saige_grm* h) {
  return align256((size_t)h->n_pad * sizeof(float)) + align256((size_t)h->m_pad * sizeof(float)) +
         (size_t)h->n_splits * h->n_pad * sizeof(float);
}

Status matvec_noalloc(saige_grm* h, const double* v, double* out, int64_t n, int nrhs,
                      cudaStream_t st) {
  if (h->m_eff == 0) {  // pcg.rs:132-134: no markers -> zero vector
    SG_CUDA(cudaMemsetAsync(out, 0, (size_t)n * nrhs * sizeof(double), st));
    return Status();
  }
  const size_t v_bytes = align256((size_t)h->n_pad * sizeof(float));
  const size_t u_bytes = align256((size_t)h->m_pad * sizeof(float));
  const size_t need = noalloc_bytes(h);
  if (need > kNoAllocScratchBytes)
    return fail(SAIGE_EINVAL,
                "saige_grm_matvec_dev_noalloc: this GRM (n=%lld, m=%lld) needs %zu bytes of "
                "scratch, above the %zu-byte static maximum; use saige_grm_matvec_dev",
                (long long)h->n, (long long)h->m, need, kNoAllocScratchBytes);
  void* base = nullptr;
  SG_TRY(scratch_address(h->device, &base));
  float* v32 = reinterpret_cast<float*>(base);
  float* u32 = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + v_bytes);
  float* ypart = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + v_bytes + u_bytes);
  const float scale = 1.0f / (float)h->m_eff;
  for (int c = 0; c < nrhs; ++c) {
    const double* vc = v + (int64_t)c * n;
    double* oc = out + (int64_t)c * n;
    // to_f32 writes all n_pad entries (zeros past n); pass A writes all m_pad
    // entries of u; pass B writes every split's plane for the sample windows that
    // the finish kernel reads.
    SG_CUDA(launch_to_f32(vc, n, h->n_pad, v32, st));
    SG_CUDA(launch_fp32_zt(h->geno, h->wpr, h->zlut, h->m_pad, v32, u32, st));
    SG_CUDA(launch_fp32_z(h->geno, h->wpr, h->zlut, h->m_pad, u32, ypart, h->n_splits, st));
    SG_CUDA(launch_fp32_finish(ypart, h->n_splits, h->n_pad, n, scale, oc, st));
  }
  h->n_kv += nrhs;
  h->n_kv_launches += 1;
  h->stats.fp32_launches += nrhs;
  return Status();
}

}  // namespace
}  // namespace saige

using namespace saige;

extern "C" __attribute__((visibility("default"))) int32_t saige_grm_matvec_dev_noalloc(
    saige_grm* h, const double* v_dev, double* out_dev, int64_t n, int32_t nrhs, void* stream) {
  try {
    set_error("");
    if (!h || !v_dev || !out_dev) return fail(SAIGE_EINVAL, "null argument").code;
    if (n != h->n) return fail(SAIGE_EINVAL, "n mismatch (%lld vs %lld)", (long long)n,
                               (long long)h->n).code;
    if (nrhs <= 0) return fail(SAIGE_EINVAL, "nrhs must be positive").code;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    DeviceGuard dg(h->device);
    if (!dg.ok) return fail(SAIGE_ECUDA, "cannot make device %d current", h->device).code;
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    return matvec_noalloc(h, v_dev, out_dev, n, nrhs, st).code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}

extern "C" __attribute__((visibility("default"))) int32_t saige_grm_noalloc_scratch_bytes(
    const saige_grm* h, size_t* need, size_t* limit) {
  set_error("");
  if (!h) return fail(SAIGE_EINVAL, "null argument").code;
  if (need) *need = noalloc_bytes(h);
  if (limit) *limit = kNoAllocScratchBytes;
  return SAIGE_OK;
}
