// Launch wrappers of the library's kernels (all sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace saige {

// ---- K1: .bed gather / repack and per-marker counts ------------------------
// For each selected row r: src marker src_rows[r] of the raw .bed (header at
// bed[0]), samples gathered in sample_idx order (NULL = identity).  When
// geno_out != NULL the 2-bit codes are written to row r of geno_out (pitch
// words_per_row 32-bit words; padding samples coded 01 = missing).  counts
// (2 per row, may be NULL) receive {alt-allele count, missing count}.
cudaError_t launch_bed_gather(const uint8_t* bed, int64_t bytes_per_marker, const int64_t* src_rows,
                              int64_t n_rows, const int32_t* sample_idx, int64_t n,
                              uint32_t* geno_out, int64_t words_per_row, int64_t* counts,
                              cudaStream_t st);

// Alt-allele and missing counts of rows j0 .. j0 + n_rows of the raw .bed for several
// sample subsets at once: subset c is sidx[offs[c] .. offs[c] + ns[c]) (offs[c] a
// multiple of 16); counts[(c m_tot + j) 2 + {0, 1}].  Rows of more than 200 KB are
// refused (cudaErrorInvalidValue).
cudaError_t launch_bed_count_cohorts(const uint8_t* bed, int64_t bytes_per_marker, int64_t j0,
                                     int64_t n_rows, const int32_t* sidx, const int64_t* offs,
                                     const int64_t* ns, int n_cohorts, int64_t m_tot,
                                     long long* counts, cudaStream_t st);

// One cohort's output of launch_bed_gather_cohorts: raw marker j goes to row
// row_of[j * row_stride] of geno (wpr words per row; -1: not kept), its n samples at
// sidx[sidx_off ..] (sidx_off a multiple of 16).  row_of may be host-mapped memory.
struct CohortRows {
  uint32_t* geno;
  const int32_t* row_of;
  int64_t row_stride;
  int64_t wpr;
  int64_t n;
  int64_t sidx_off;
};
// Up to kCohortsPerLaunch cohorts, passed by value in the launch's parameters (no copy
// to queue behind other transfers).
constexpr int kCohortsPerLaunch = 32;
struct CohortSet {
  CohortRows c[kCohortsPerLaunch];
  int n;
};
// Gathers raw rows j0 .. j0 + n_rows into every cohort of the set that keeps them.  Rows
// of more than 200 KB are refused.
cudaError_t launch_bed_gather_cohorts(const uint8_t* bed, int64_t bytes_per_marker, int64_t j0,
                                      int64_t n_rows, const int32_t* sidx, const CohortSet& set,
                                      cudaStream_t st);

// ---- synthetic cohort ------------------------------------------------------
struct CohortDev;
cudaError_t launch_gen_bed(const void* layout, uint8_t* bed, int64_t bytes_per_marker,
                           int64_t m, cudaStream_t st);

// ---- FP32 GRM product (saige-rs arithmetic) --------------------------------
// u[m] = sum_i z(code_mi) v32[i]       (pass A, f32)
cudaError_t launch_fp32_zt(const uint32_t* geno, int64_t words_per_row, const float4* zlut,
                           int64_t m_pad, const float* v32, float* u, cudaStream_t st);
// ypart[s][i] = sum_{m in split s} z(code_mi) u[m]   (pass B, f32)
cudaError_t launch_fp32_z(const uint32_t* geno, int64_t words_per_row, const float4* zlut,
                          int64_t m_pad, const float* u, float* ypart, int n_splits,
                          cudaStream_t st);
int fp32_z_splits(int64_t n_pad, int64_t m_pad);
// out[i] = (double)((sum_s ypart[s][i]) * scale)  (f32 arithmetic)
cudaError_t launch_fp32_finish(const float* ypart, int n_splits, int64_t n_pad, int64_t n,
                               float scale, double* out, cudaStream_t st);
// v32[i] = (float)v[i] for i < n, 0 for n <= i < n_pad
cudaError_t launch_to_f32(const double* v, int64_t n, int64_t n_pad, float* v32,
                          cudaStream_t st);

}  // namespace saige
