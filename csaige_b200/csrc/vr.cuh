// Variance ratio inside the fit-null pipeline (vr.cu).
#pragma once
#include "engine.cuh"

namespace saige {

// Packed .bed rows of the variance-ratio candidates, kept on the device after
// the full .bed is released.
struct VrRows {
  DevBuf rows;  // m x bpm bytes
  DevBuf sidx;  // sample subset (n int64), when given
  int64_t bpm = 0, m = 0;
  bool has_sidx = false;
};

// Copies the rows vidx[0..m_vr) of a device .bed (bed_dev points at the header).
Status vr_gather_rows(const uint8_t* bed_dev, int64_t bpm, const int64_t* vidx, int64_t m_vr,
                      const int64_t* sample_idx, int64_t n, VrRows& out, cudaStream_t st);

// estimate_variance_ratio over those rows (mac per row), as fit_null.rs:290-373.
Status vr_from_rows(saige_grm* h, const VrRows& rows, const double* mac, const double* mu,
                    const double* w, const double tau[2], int trait, const double* x, int p,
                    const saige_vr_config* cfg, saige_vr_summary* out);

}  // namespace saige
