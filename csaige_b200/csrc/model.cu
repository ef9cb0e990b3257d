// The .saige.model writer: NullModel (saige-core/src/model/null_model.rs:17-113)
// serialised as saige-rs does it, bincode::serialize (serialization.rs:13-17).
//
// bincode 1.3.3 with its default options writes the struct's fields in
// declaration order with fixed-width little-endian integers: u32/u64 as 4/8
// bytes, usize as u64, f64 as its 8 IEEE bytes, bool as one byte, a fixed array
// ([u8; 4], [f64; 2]) as its elements, a String or Vec as a u64 length followed
// by the bytes or elements, a tuple as its elements, and a unit enum variant
// (TraitType) as its u32 index.
#include <stdint.h>
#include <string.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "common.cuh"

namespace saige {
namespace {

struct Writer {
  std::vector<uint8_t> b;
  void u8(uint8_t v) { b.push_back(v); }
  void u32(uint32_t v) {
    for (int i = 0; i < 4; ++i) b.push_back((uint8_t)(v >> (8 * i)));
  }
  void u64(uint64_t v) {
    for (int i = 0; i < 8; ++i) b.push_back((uint8_t)(v >> (8 * i)));
  }
  void f64(double v) {
    uint64_t u;
    memcpy(&u, &v, 8);
    u64(u);
  }
  void str(const char* s) {
    const size_t n = strlen(s);
    u64(n);
    b.insert(b.end(), s, s + n);
  }
  void vec(const double* v, int64_t n) {
    u64((uint64_t)n);
    for (int64_t i = 0; i < n; ++i) f64(v[i]);
  }
};

}  // namespace
}  // namespace saige

using namespace saige;

#define SG_API extern "C" __attribute__((visibility("default")))

SG_API int32_t saige_xvx_inv_xv(const double* x, const double* w, int64_t n, int32_t p,
                                double* out) {
  try {
    set_error("");
    if (!x || !w || !out || n <= 0 || p <= 0 || p > 64)
      return fail(SAIGE_EINVAL, "null argument or bad size").code;
    // fit_null.rs:291: XVX = X'WX (dense.rs:227-245)
    std::vector<double> xvx((size_t)p * p), l((size_t)p * p, 0.0), inv((size_t)p * p);
    for (int j = 0; j < p; ++j)
      for (int k = j; k < p; ++k) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += x[(int64_t)j * n + i] * w[i] * x[(int64_t)k * n + i];
        xvx[(size_t)j * p + k] = s;
        xvx[(size_t)k * p + j] = s;
      }
    // inverse_spd (decomposition.rs:362-365): Cholesky (35-62), unit-column solves (64-102)
    for (int j = 0; j < p; ++j) {
      double sum = 0.0;
      for (int k = 0; k < j; ++k) sum += l[(size_t)j * p + k] * l[(size_t)j * p + k];
      const double diag = xvx[(size_t)j * p + j] - sum;
      if (diag <= 0.0) return fail(SAIGE_SINGULAR, "Matrix is not positive definite").code;
      l[(size_t)j * p + j] = std::sqrt(diag);
      for (int i = j + 1; i < p; ++i) {
        double s = 0.0;
        for (int k = 0; k < j; ++k) s += l[(size_t)i * p + k] * l[(size_t)j * p + k];
        l[(size_t)i * p + j] = (xvx[(size_t)i * p + j] - s) / l[(size_t)j * p + j];
      }
    }
    for (int c = 0; c < p; ++c) {
      std::vector<double> y((size_t)p), xs((size_t)p);
      for (int i = 0; i < p; ++i) {
        double s = 0.0;
        for (int j = 0; j < i; ++j) s += l[(size_t)i * p + j] * y[(size_t)j];
        y[(size_t)i] = ((i == c ? 1.0 : 0.0) - s) / l[(size_t)i * p + i];
      }
      for (int i = p - 1; i >= 0; --i) {
        double s = 0.0;
        for (int j = i + 1; j < p; ++j) s += l[(size_t)j * p + i] * xs[(size_t)j];
        xs[(size_t)i] = (y[(size_t)i] - s) / l[(size_t)i * p + i];
      }
      for (int k = 0; k < p; ++k) inv[(size_t)k * p + c] = xs[(size_t)k];
    }
    // fit_null.rs:294-305: data[j*n + i] = sum_k inv(j,k) x(i,k) w(i)
    for (int j = 0; j < p; ++j)
      for (int64_t i = 0; i < n; ++i) {
        double val = 0.0;
        for (int k = 0; k < p; ++k) val += inv[(size_t)j * p + k] * x[(int64_t)k * n + i] * w[i];
        out[(int64_t)j * n + i] = val;
      }
    return SAIGE_OK;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}

SG_API int32_t saige_write_null_model(const char* path, const saige_null_model* m) {
  try {
    set_error("");
    if (!path || !m || !m->alpha || !m->mu || !m->y || !m->x || !m->xvx_inv_xv)
      return fail(SAIGE_EINVAL, "null argument").code;
    if (m->trait < 0 || m->trait > 2) return fail(SAIGE_EINVAL, "unknown trait type").code;
    if (m->n < 0 || m->p <= 0) return fail(SAIGE_EINVAL, "bad dimensions").code;
    if (m->n > 0 && !m->sample_ids) return fail(SAIGE_EINVAL, "sample_ids missing").code;
    if (m->n_loco > 0 && (!m->loco_chrom || !m->loco_tau || !m->loco_mu || !m->loco_residuals))
      return fail(SAIGE_EINVAL, "LOCO arrays missing").code;
    const int64_t n = m->n, p = m->p;
    Writer w;
    // magic "SGMD", version 1 (null_model.rs:64-67)
    for (char c : std::string("SGMD")) w.u8((uint8_t)c);
    w.u32(1);
    w.u32((uint32_t)m->trait);  // TraitType variant index: Binary 0, Quantitative 1, Survival 2
    w.u64((uint64_t)n);          // sample_ids
    for (int64_t i = 0; i < n; ++i) w.str(m->sample_ids[i]);
    w.u64((uint64_t)n);  // n_samples
    w.u64((uint64_t)p);  // n_covariates
    w.f64(m->tau[0]);
    w.f64(m->tau[1]);
    w.vec(m->alpha, p);
    w.vec(m->mu, n);
    // mu2 and residuals as NullModel::new computes them (null_model.rs:83-88)
    w.u64((uint64_t)n);
    for (int64_t i = 0; i < n; ++i)
      w.f64(m->trait == SAIGE_TRAIT_QUANTITATIVE ? 1.0 : m->mu[i] * (1.0 - m->mu[i]));
    w.u64((uint64_t)n);
    for (int64_t i = 0; i < n; ++i) w.f64(m->y[i] - m->mu[i]);
    w.vec(m->y, n);
    w.vec(m->x, n * p);  // x_flat, column-major n x p
    w.u64((uint64_t)p);  // x_ncols
    w.vec(m->xvx_inv_xv, p * n);
    // VarianceRatioResult (variance_ratio.rs:59-71)
    w.f64(m->variance_ratio);
    w.u64((uint64_t)m->vr_n_categories);
    for (int32_t k = 0; k < m->vr_n_categories; ++k) {
      w.f64(m->vr_cat_upper[k]);
      w.f64(m->vr_cat_vr[k]);
    }
    w.u64((uint64_t)m->vr_n_markers_used);
    w.vec(m->vr_per_marker ? m->vr_per_marker : nullptr, m->vr_per_marker ? m->vr_n_per_marker : 0);
    w.u8(m->use_loco ? 1 : 0);
    w.u64((uint64_t)m->n_loco);  // loco_tau: Vec<(String, [f64; 2])>
    for (int32_t k = 0; k < m->n_loco; ++k) {
      w.str(m->loco_chrom[k]);
      w.f64(m->loco_tau[2 * k]);
      w.f64(m->loco_tau[2 * k + 1]);
    }
    w.u64((uint64_t)m->n_loco);  // loco_mu: Vec<(String, Vec<f64>)>
    for (int32_t k = 0; k < m->n_loco; ++k) {
      w.str(m->loco_chrom[k]);
      w.vec(m->loco_mu + (int64_t)k * n, n);
    }
    w.u64((uint64_t)m->n_loco);  // loco_residuals
    for (int32_t k = 0; k < m->n_loco; ++k) {
      w.str(m->loco_chrom[k]);
      w.vec(m->loco_residuals + (int64_t)k * n, n);
    }
    w.u8(m->use_sparse_grm ? 1 : 0);
    w.u64((uint64_t)m->n_markers_in_grm);
    FILE* f = fopen(path, "wb");
    if (!f) return fail(SAIGE_EINVAL, "cannot open %s for writing", path).code;
    const size_t put = fwrite(w.b.data(), 1, w.b.size(), f);
    const int cl = fclose(f);
    if (put != w.b.size() || cl != 0) return fail(SAIGE_EINVAL, "writing %s failed", path).code;
    return SAIGE_OK;
  } catch (const std::bad_alloc&) {
    return fail(SAIGE_ENOMEM, "host allocation failed").code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}
