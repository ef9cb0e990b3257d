// AI-REML fit of the null GLMM on the GPU: fit_ai_reml and fit_glm_irls of
// saige-core/src/glmm/ai_reml.rs:86-482.  N-vectors stay in HBM; the p x p
// Cholesky solves (p <= 64) and the tau update run on the host in FP64.
#include <math.h>
#include <string.h>

#include <cstdlib>
#include <chrono>
#include <thread>
#include <vector>

#include "engine.cuh"
#include "kernels_tc.cuh"
#include "kernels.cuh"
#include "rng.hpp"
#include "vr.cuh"
#include "mlp.cuh"
#include "warm.cuh"

namespace saige {

namespace {

// decomposition.rs:35-61 (row-major p x p); false when not positive definite.
bool cholesky(const std::vector<double>& a, int p, std::vector<double>& l) {
  l.assign((size_t)p * p, 0.0);
  for (int j = 0; j < p; ++j) {
    double sum = 0.0;
    for (int k = 0; k < j; ++k) sum += l[j * p + k] * l[j * p + k];
    const double diag = a[j * p + j] - sum;
    if (diag <= 0.0) return false;
    l[j * p + j] = sqrt(diag);
    for (int i = j + 1; i < p; ++i) {
      double s = 0.0;
      for (int k = 0; k < j; ++k) s += l[i * p + k] * l[j * p + k];
      l[i * p + j] = (a[i * p + j] - s) / l[j * p + j];
    }
  }
  return true;
}

// decomposition.rs:64-89
void chol_solve(const std::vector<double>& l, int p, const double* b, double* x) {
  std::vector<double> y((size_t)p);
  for (int i = 0; i < p; ++i) {
    double s = 0.0;
    for (int j = 0; j < i; ++j) s += l[i * p + j] * y[j];
    y[i] = (b[i] - s) / l[i * p + i];
  }
  for (int i = p - 1; i >= 0; --i) {
    double s = 0.0;
    for (int j = i + 1; j < p; ++j) s += l[j * p + i] * x[j];
    x[i] = (y[i] - s) / l[i * p + i];
  }
}

struct Fit {
  saige_grm* h;
  cudaStream_t st;
  int64_t n, ld;
  int p, nrv, q;
  const saige_ai_reml_config* cfg;
  DevBuf mem;
  // device vectors
  double *y, *x, *eta, *mu, *w, *wmax, *d, *ytil;
  double *rhs, *sol;      // n_pad x q each: [ytil | X | U], [Sinv ytil | Sinv X | Sinv U]
  double *kxu, *ku, *pu, *tmpq; // K [X | U] (n_pad x (p + nrv)); ku = its U part; n_pad x nrv
  double *py, *kpy, *pk, *invw_py, *pw, *pk_raw, *pw_raw;
  double *dsmall;         // small device scratch (coefficients, dot results)
  double *partial;
  int64_t pcg_iters = 0;
  bool have_prev = false, have_prev_pk = false, have_prev_pw = false;
};

Status dots(Fit& f, const double* a, int pa, const double* b, int qb, const double* wv,
            std::vector<double>& out) {
  double* dout = f.dsmall;
  SG_CUDA(cross_dots(a, pa, b, qb, wv, f.n, f.ld, f.partial, dout, f.st));
  out.resize((size_t)pa * qb);
  SG_CUDA(cudaMemcpyAsync(out.data(), dout, out.size() * 8, cudaMemcpyDeviceToHost, f.st));
  SG_CUDA(cudaStreamSynchronize(f.st));
  return Status();
}

Status coldots(Fit& f, const double* a, const double* b, int q, std::vector<double>& out) {
  double* dout = f.dsmall;
  SG_CUDA(col_dots(a, b, f.n, f.ld, q, f.partial, dout, f.st));
  out.resize((size_t)q);
  SG_CUDA(cudaMemcpyAsync(out.data(), dout, out.size() * 8, cudaMemcpyDeviceToHost, f.st));
  SG_CUDA(cudaStreamSynchronize(f.st));
  return Status();
}

// PCG of Sigma = tau0 W^-1 + tau1 K on q columns of b into x (x0 optional).
struct Extra {
  const double* in = nullptr;
  double* out = nullptr;
  int n = 0;
};
// search directions of the leading columns kept by the solve (with K-images)
struct Keep {
  double* p = nullptr;
  double* kp = nullptr;
  int cols = 0, cap = 0, kept = 0;
};

Status solve(Fit& f, const double* b, double* x, const double* x0, int q, const double tau[2],
             const double* ax0 = nullptr, double* r_out = nullptr, double* kx = nullptr,
             const double* kx0 = nullptr, bool* kx_valid = nullptr, Extra extra = Extra(),
             Keep* keep = nullptr) {
  PcgRun run;
  run.b = b;
  run.x0 = x0;
  run.ax0 = x0 ? ax0 : nullptr;
  run.r_out = r_out;
  run.kx = kx;
  run.kx0 = x0 ? kx0 : nullptr;
  run.extra_in = extra.in;
  run.extra_out = extra.out;
  run.n_extra = extra.n;
  run.wv = f.wmax;
  run.d = f.d;
  run.tau0 = tau[0];
  run.tau1 = tau[1];
  run.q = q;
  run.tol = f.cfg->pcg_tol;
  run.max_iter = f.cfg->pcg_max_iter;
  run.precision = f.cfg->precision;
  run.x = x;
  // A warm-started column takes at least one step even when its start meets the
  // tolerance (the reference, starting from zero, always refines against the current
  // operator).  Measured at N = 200k, M = 150k, τ tolerance 1e-5: without the step the fit
  // launched 8 products instead of 10, but took 10 AI-REML iterations instead of 5 and
  // ended 3.4e-4 away in tau1.
  run.force_step = x0 != nullptr;
  if (keep) {
    run.keep_p = keep->p;
    run.keep_kp = keep->kp;
    run.keep_cols = keep->cols;
    run.keep_cap = keep->cap;
  }
  SG_TRY(pcg_run(f.h, run, f.st));
  if (keep) keep->kept = run.kept;
  f.pcg_iters += run.total_iters;
  if (kx_valid) *kx_valid = run.kx_valid;
  return Status();
}

// P-projection (ai_reml.rs:242-251) of q solved columns sol (in place):
// sol -= SinvX C^-1 (SinvX' u).
Status p_project(Fit& f, double* sol, const double* u, int q, const std::vector<double>& l) {
  std::vector<double> t;
  SG_TRY(dots(f, f.sol + f.ld, f.p, u, q, nullptr, t));  // p x q
  std::vector<double> coef((size_t)f.p * q), col((size_t)f.p), corr((size_t)f.p);
  for (int c = 0; c < q; ++c) {
    for (int j = 0; j < f.p; ++j) col[(size_t)j] = t[(size_t)j * q + c];
    chol_solve(l, f.p, col.data(), corr.data());
    for (int j = 0; j < f.p; ++j) coef[(size_t)j * q + c] = corr[(size_t)j];
  }
  SG_CUDA(cudaMemcpyAsync(f.dsmall, coef.data(), coef.size() * 8, cudaMemcpyHostToDevice, f.st));
  SG_CUDA(sub_combo(sol, q, f.sol + f.ld, f.p, f.dsmall, f.n, f.ld, f.st));
  return Status();
}

Status copy_cols(Fit& f, const double* src, double* dst, int q) {
  SG_CUDA(cudaMemcpyAsync(dst, src, (size_t)f.ld * q * 8, cudaMemcpyDeviceToDevice, f.st));
  return Status();
}

// ---- recycled starts -------------------------------------------------------
// A start x0 = V g with Sigma x0 = (Sigma V) g known needs no GRM product for its
// residual.  V holds vectors whose Sigma-image is known without a product of its
// own: X and the probes U (K X and K U come from one launch per fit), the block
// solutions of the previous iteration and the previous AI solutions (their K-images
// ride in the K Py launch, whose cost hardly grows with the column count), and, for
// the AI solves, this iteration's block solutions (Sigma x = b - r exactly).
// g solves the Galerkin system (V' Sigma V) g = V' b, the start of least
// Sigma-norm error in span V; the solve is then an ordinary PCG from x0.
struct Recycle {
  int mb_max = 0, nk = 0;
  DevBuf mem;                           // one block (large blocks are cached)
  double *v, *av, *x0, *ax0, *br;       // basis, images (+ b), start, its image, block r
  double *kv, *kx0;                     // K-images of the basis columns and of the start
  double *kblock, *kpk, *kpw;           // K X* of the latest block solve, K of the AI solutions
  double *kin, *kout;                   // [Py | X*_t | pk' | pw' (| learned)] and its K-image
  double *gam, *gpart, *gout;
  bool have_kblock = false, have_kpk = false, have_kpw = false;
  bool kv_ok = true;                    // every basis column of the current start has kv
  // K [X | U] was formed (f.kxu).  Without it (the recycled block fit) [X | U] joins a
  // basis only while tau1 = 0, where its Sigma-image needs no K, and the Hutchinson
  // trace takes K P u from the block solutions' K-images.
  bool kxu_ok = true;
  // the block solve's search directions of its y and X columns with their K-images
  // (a Krylov basis for K P y, whose Sigma^-1-image the AI solve wants); valid as
  // basis vectors at any tau since their Sigma-images come from the K-images
  double *keep_p = nullptr, *keep_kp = nullptr;
  int keep_cap = 0, n_keep = 0;
  bool with_pw = false;                 // the fit has the W^-1 AI solve (quantitative)
  int64_t fallbacks = 0, kpy_launches_saved = 0;
  // learned correction (SAIGE_WARM_LEARNED): an MLP trained on the change of the
  // block solutions between iterations predicts the next change; the prediction joins
  // the next block basis, its K-image from the K Py launch
  bool learned = false;
  Mlp mlp;
  DevBuf lmem;
  float *F0 = nullptr, *F1 = nullptr, *T = nullptr, *yhat = nullptr;
  double *xprev = nullptr, *delta = nullptr, *bnext = nullptr, *wnext = nullptr, *scales = nullptr;
  const double* diagk = nullptr;
  bool have_F = false, have_delta = false;
  int at_delta = 0, trainings = 0, uses = 0;
  double r2 = 0.0, seconds = 0.0;
};

// Held-out R^2 at or above which the prediction joins the basis.
constexpr double kLearnR2Min = 0.25;
// Adam steps of the first and of every later training round, and the learning rate.
constexpr int kLearnSteps0 = 100;
constexpr int kLearnSteps = 50;
constexpr float kLearnRate = 1e-3f;
// PCG iterations of the block solve whose y and X search directions are kept
constexpr int kKeepIters = 3;
// At most this many kept directions (each costs two n-vectors of workspace plus a
// column of every recycled basis and Galerkin system): the first kKeepIters
// iterations of y and up to 15 covariates; with more covariates the later columns'
// directions are not kept.
constexpr int kKeepMaxCols = 48;

Status recycle_init(Fit& f, Recycle& rc, bool learned, const double* diagk, uint64_t seed) {
  const size_t ld = (size_t)f.ld, q = (size_t)f.q;
  rc.learned = learned;
  rc.diagk = diagk;
  rc.keep_cap = std::min((1 + f.p) * kKeepIters, kKeepMaxCols);
  rc.mb_max = (learned ? 3 * f.q + 1 : 2 * f.q + 1) + rc.keep_cap;
  rc.nk = learned ? 2 * f.q + 3 : f.q + 3;
  if (learned) {
    const size_t nq = (size_t)f.n * q;
    SG_TRY(rc.lmem.reserve(nq * (2 * kMlpIn + 2) * 4 + (3 * q + 1) * ld * 8 + (2 * q + 8) * 8 + 64));
    char* c = rc.lmem.as<char>();
    rc.xprev = reinterpret_cast<double*>(c);
    rc.delta = rc.xprev + q * ld;
    rc.bnext = rc.delta + q * ld;
    rc.wnext = rc.bnext + q * ld;
    rc.scales = rc.wnext + ld;
    rc.F0 = reinterpret_cast<float*>(rc.scales + 2 * q + 8);
    rc.F1 = rc.F0 + nq * kMlpIn;
    rc.T = rc.F1 + nq * kMlpIn;
    rc.yhat = rc.T + nq;
    SG_CUDA(cudaMemsetAsync(rc.xprev, 0, (3 * q + 1) * ld * 8, f.st));
    SG_TRY(mlp_init(rc.mlp, seed, f.st));
  }
  const size_t mb = (size_t)rc.mb_max, nk = (size_t)rc.nk;
  const size_t ncol = mb + (mb + q) + 3 * q + 2 * nk + mb + q + q + 2 + 2 * (size_t)rc.keep_cap;
  const size_t nsmall = mb * q + gram_partial_doubles(f.n, (int)mb, (int)(mb + q)) + mb * (mb + q);
  SG_TRY(rc.mem.reserve((ncol * ld + nsmall) * 8));
  double* b = rc.mem.as<double>();
  SG_CUDA(cudaMemsetAsync(b, 0, ncol * ld * 8, f.st));  // padding rows stay zero
  rc.v = b;                 b += mb * ld;
  rc.av = b;                b += (mb + q) * ld;
  rc.x0 = b;                b += q * ld;
  rc.ax0 = b;               b += q * ld;
  rc.br = b;                b += q * ld;
  rc.kin = b;               b += nk * ld;
  rc.kout = b;              b += nk * ld;
  rc.kv = b;                b += mb * ld;
  rc.kx0 = b;               b += q * ld;
  rc.kblock = b;            b += q * ld;
  rc.kpk = b;               b += ld;
  rc.kpw = b;               b += ld;
  rc.keep_p = b;            b += (size_t)rc.keep_cap * ld;
  rc.keep_kp = b;           b += (size_t)rc.keep_cap * ld;
  rc.gam = b;               b += mb * q;
  rc.gout = b;              b += mb * (mb + q);
  rc.gpart = b;
  return Status();
}

// Coefficients g (mb x q, row-major) of (V' A V) g = V' B from the Gram block
// gall = V' [A V | B] (mb x (mb + q)): Jacobi-scaled, with the smallest ridge
// (relative 1e-12 .. 1e-6) under which the Cholesky factorisation succeeds.
bool galerkin_coeffs(const std::vector<double>& gall, int mb, int q, std::vector<double>& gam) {
  const int w = mb + q;
  std::vector<double> s((size_t)mb), a((size_t)mb * mb), l;
  for (int i = 0; i < mb; ++i) {
    const double d = gall[(size_t)i * w + i];
    s[(size_t)i] = (d > 0.0 && std::isfinite(d)) ? 1.0 / sqrt(d) : 0.0;
  }
  bool ok = false;
  for (double ridge : {1e-12, 1e-10, 1e-8, 1e-6}) {
    for (int i = 0; i < mb; ++i)
      for (int j = 0; j < mb; ++j) {
        double v = 0.5 * (gall[(size_t)i * w + j] + gall[(size_t)j * w + i]) * s[(size_t)i] *
                   s[(size_t)j];
        if (i == j) v = (s[(size_t)i] > 0.0 ? v : 1.0) + ridge;
        a[(size_t)i * mb + j] = v;
      }
    if (cholesky(a, mb, l)) {
      ok = true;
      break;
    }
  }
  if (!ok) return false;
  gam.assign((size_t)mb * q, 0.0);
  std::vector<double> rhs((size_t)mb), y((size_t)mb);
  for (int c = 0; c < q; ++c) {
    for (int i = 0; i < mb; ++i) rhs[(size_t)i] = s[(size_t)i] * gall[(size_t)i * w + mb + c];
    chol_solve(l, mb, rhs.data(), y.data());
    for (int i = 0; i < mb; ++i) {
      const double g = s[(size_t)i] * y[(size_t)i];
      if (!std::isfinite(g)) return false;
      gam[(size_t)i * q + c] = g;
    }
  }
  return true;
}

// With rc.v[0..mb) and rc.av[0..mb) filled and b (q columns) at rc.av[mb..mb+q):
// x0 = V g into rc.x0 and Sigma x0 into rc.ax0; ok = false when the projected system
// cannot be factorised (no start).
Status galerkin_start(Fit& f, Recycle& rc, int mb, int q, bool& ok) {
  const int64_t ld = f.ld;
  SG_CUDA(gram(rc.v, mb, rc.av, mb + q, f.n, ld, rc.gpart, rc.gout, f.st));
  std::vector<double> gall((size_t)mb * (mb + q)), gam;
  SG_CUDA(cudaMemcpyAsync(gall.data(), rc.gout, gall.size() * 8, cudaMemcpyDeviceToHost, f.st));
  SG_CUDA(cudaStreamSynchronize(f.st));
  ok = galerkin_coeffs(gall, mb, q, gam);
  if (!ok) {
    ++rc.fallbacks;
    return Status();
  }
  SG_CUDA(cudaMemcpyAsync(rc.gam, gam.data(), gam.size() * 8, cudaMemcpyHostToDevice, f.st));
  SG_CUDA(combo(rc.v, mb, rc.gam, q, rc.x0, false, f.n, ld, f.st));
  SG_CUDA(combo(rc.av, mb, rc.gam, q, rc.ax0, false, f.n, ld, f.st));
  if (rc.kv_ok) SG_CUDA(combo(rc.kv, mb, rc.gam, q, rc.kx0, false, f.n, ld, f.st));
  return Status();
}

// k basis columns x with K-images kx, and their images under the current Sigma,
// at column `at` of rc.v / rc.av.
Status basis_cols(Fit& f, Recycle& rc, int at, const double* x, const double* kx, int k,
                  const double tau[2]) {
  const int64_t ld = f.ld;
  if (at + k > rc.mb_max) return fail(SAIGE_EINVAL, "start basis beyond its %d columns", rc.mb_max);
  SG_TRY(copy_cols(f, x, rc.v + (size_t)at * ld, k));
  SG_TRY(copy_cols(f, kx, rc.kv + (size_t)at * ld, k));
  SG_CUDA(sigma_image(x, kx, f.wmax, tau[0], tau[1], rc.av + (size_t)at * ld, f.n, ld, k, f.st));
  return Status();
}

// The block solve of one iteration from the recycled start: basis [X | U] and the
// previous iteration's block solutions (f.sol on entry, K-image rc.kblock).  Leaves the
// final residual in rc.br and K X*_t in rc.kblock; kx_ok tells whether that K-image was
// formed (false when the iteration has tau1 = 0, whose solve forms no product).
Status block_solve_recycled(Fit& f, Recycle& rc, const double* x0_prev, const double tau[2],
                            bool& kx_ok) {
  const int64_t ld = f.ld;
  int mb = 0;
  rc.kv_ok = true;
  if (rc.kxu_ok || tau[1] == 0.0) {
    SG_TRY(basis_cols(f, rc, mb, f.rhs + ld, f.kxu, f.p + f.nrv, tau));
    mb += f.p + f.nrv;
    if (!rc.kxu_ok) rc.kv_ok = false;  // zero stand-ins for K [X | U]: no K x0
  }
  if (rc.have_kblock) {
    SG_TRY(basis_cols(f, rc, mb, f.sol, rc.kblock, f.q, tau));
    mb += f.q;
  }
  if (rc.n_keep > 0) {  // the previous block solve's directions (their K-images known)
    SG_TRY(basis_cols(f, rc, mb, rc.keep_p, rc.keep_kp, rc.n_keep, tau));
    mb += rc.n_keep;
  }
  if (rc.have_delta) {
    // the learned prediction of this iteration's change of the solutions
    SG_TRY(basis_cols(f, rc, mb, rc.delta, rc.kout + (size_t)rc.at_delta * ld, f.q, tau));
    mb += f.q;
    ++rc.uses;
  }
  SG_TRY(copy_cols(f, f.rhs, rc.av + (size_t)mb * ld, f.q));
  bool ok = false;
  SG_TRY(galerkin_start(f, rc, mb, f.q, ok));
  kx_ok = false;
  // the previous AI solutions whose K-image is missing (their solve had tau1 = 0) ride
  // in the first product of this solve, for this iteration's AI starts
  Extra ex;
  if (!rc.learned && tau[1] != 0.0) {
    // (measured: leaving them out to keep this product at kTcFastCols columns cost the
    // AI solve one more product than the slower launch shape costs)
    const bool need_pk = f.have_prev_pk && !rc.have_kpk;
    const bool need_pw = rc.with_pw && f.have_prev_pw && !rc.have_kpw;
    if (need_pk && need_pw) ex = Extra{f.pk_raw, rc.kpk, 2};  // adjacent columns
    else if (need_pk) ex = Extra{f.pk_raw, rc.kpk, 1};
    else if (need_pw) ex = Extra{f.pw_raw, rc.kpw, 1};
    if (need_pk) rc.have_kpk = true;
    if (need_pw) rc.have_kpw = true;
  }
  // keep this solve's y and X directions (overwriting the ones copied into the basis)
  Keep keep{rc.keep_p, rc.keep_kp, 1 + f.p, rc.keep_cap, 0};
  Status s = ok ? solve(f, f.rhs, f.sol, rc.x0, f.q, tau, rc.ax0, rc.br, rc.kblock,
                        rc.kv_ok ? rc.kx0 : nullptr, &kx_ok, ex, &keep)
                : solve(f, f.rhs, f.sol, x0_prev, f.q, tau, nullptr, rc.br, rc.kblock, nullptr,
                        &kx_ok, ex, &keep);
  if (tau[1] != 0.0) rc.n_keep = keep.kept;  // with tau1 = 0 the solve forms no K-images
  return s;
}

// K Py = K (Sinv y - Sinv X alpha) = kblock[:, 0] - kblock[:, 1..p] alpha from the
// K-images of this iteration's block solutions (alpha uploaded again: the device
// scratch also takes dot results).
Status kpy_combine(Fit& f, Recycle& rc, const std::vector<double>& alpha) {
  SG_CUDA(cudaMemcpyAsync(f.dsmall, alpha.data(), (size_t)f.p * 8, cudaMemcpyHostToDevice, f.st));
  SG_TRY(copy_cols(f, rc.kblock, f.kpy, 1));
  SG_CUDA(sub_combo(f.kpy, 1, rc.kblock + f.ld, f.p, f.dsmall, f.n, f.ld, f.st));
  return Status();
}

// K X*_t (this iteration's block solutions, for the next block start) and K of the
// previous AI solutions pk', pw' (for this iteration's AI starts) in one launch; K Py
// then follows from K X*_t, so that the launch holds q columns (+ the AI solutions),
// not 1 + q.  Writes f.kpy.
Status learn_step(Fit& f, Recycle& rc, int trait, const double tau[2], int& k);

Status kpy_recycled(Fit& f, Recycle& rc, bool with_pk, bool with_pw, int trait,
                    const double tau[2], const std::vector<double>& alpha) {
  const int64_t ld = f.ld;
  SG_TRY(copy_cols(f, f.sol, rc.kin, f.q));
  int k = f.q;
  const int at_pk = k;
  if (with_pk) SG_TRY(copy_cols(f, f.pk_raw, rc.kin + (size_t)k++ * ld, 1));
  const int at_pw = k;
  if (with_pw) SG_TRY(copy_cols(f, f.pw_raw, rc.kin + (size_t)k++ * ld, 1));
  if (rc.learned) SG_TRY(learn_step(f, rc, trait, tau, k));
  SG_TRY(grm_product(f.h, rc.kin, rc.kout, k, nullptr, f.cfg->precision, f.st));
  SG_TRY(copy_cols(f, rc.kout, rc.kblock, f.q));
  rc.have_kblock = true;
  SG_TRY(kpy_combine(f, rc, alpha));
  if (with_pk) SG_TRY(copy_cols(f, rc.kout + (size_t)at_pk * ld, rc.kpk, 1));
  if (with_pw) SG_TRY(copy_cols(f, rc.kout + (size_t)at_pw * ld, rc.kpw, 1));
  rc.have_kpk = with_pk;
  rc.have_kpw = with_pw;
  return Status();
}

// K Py without a product: the block solve kept K X*_t beside X*_t.
Status kpy_from_block(Fit& f, Recycle& rc, const std::vector<double>& alpha) {
  SG_TRY(kpy_combine(f, rc, alpha));
  ++rc.kpy_launches_saved;
  return Status();
}

// Learned correction, at the K Py point of an iteration (block solutions X*_t in
// f.sol, the weights of the next iteration computable from the updated mu):
//  1. with the features of the previous iteration, fit the MLP to the change
//     X*_t - X*_{t-1} (per-column RMS scaled) and measure its held-out R^2;
//  2. form this iteration's features;
//  3. when the R^2 is at least kLearnR2Min, predict the next change and append it to
//     the K launch (column k on), so that the next block start may use it.
Status learn_step(Fit& f, Recycle& rc, int trait, const double tau[2], int& k) {
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t ld = f.ld, n = f.n;
  const int q = f.q;
  std::vector<double> sc((size_t)(2 * q + 8)), dd;
  if (rc.have_F) {
    SG_CUDA(sub_cols(f.sol, rc.xprev, rc.x0, n, ld, q, f.st));
    SG_TRY(coldots(f, rc.x0, rc.x0, q, dd));
    for (int c = 0; c < q; ++c) sc[(size_t)c] = sqrt(dd[(size_t)c] / (double)n);
    SG_CUDA(cudaMemcpyAsync(rc.scales, sc.data(), (size_t)q * 8, cudaMemcpyHostToDevice, f.st));
    SG_CUDA(learn_targets(f.sol, rc.xprev, rc.scales, n, ld, q, rc.T, f.st));
    SG_TRY(mlp_train(rc.mlp, rc.F0, rc.T, n, q, rc.trainings == 0 ? kLearnSteps0 : kLearnSteps,
                     kLearnRate, 8, f.st));
    double mse = 0.0, tms = 0.0;
    SG_TRY(mlp_validate(rc.mlp, rc.F0, rc.T, n, q, 8, &mse, &tms, f.st));
    rc.r2 = tms > 0.0 ? 1.0 - mse / tms : 0.0;
    ++rc.trainings;
  }
  // features of this iteration: x = X*_t, b = [ytil | X | U], bnext = next [ytil | X | U]
  SG_CUDA(work_vectors(f.y, f.eta, f.mu, trait, rc.wnext, rc.bnext, n, f.st));
  SG_TRY(copy_cols(f, f.rhs + ld, rc.bnext + ld, q - 1));
  std::vector<double> a, b, u, w;
  SG_TRY(coldots(f, f.sol, f.sol, q, a));
  SG_TRY(coldots(f, f.rhs, f.rhs, q, b));
  const int n_sk = std::min(f.nrv, 8);  // sketches: the GRM applied to the first probes
  SG_TRY(coldots(f, f.ku, f.ku, n_sk, u));
  SG_TRY(coldots(f, f.w, f.w, 1, w));
  for (int c = 0; c < q; ++c) {
    sc[(size_t)c] = sqrt(a[(size_t)c] / (double)n);
    sc[(size_t)(q + c)] = sqrt(b[(size_t)c] / (double)n);
  }
  for (int s2 = 0; s2 < 8; ++s2)
    sc[(size_t)(2 * q + s2)] = s2 < n_sk ? sqrt(u[(size_t)s2] / (double)n) : 0.0;
  const double wr = sqrt(w[0] / (double)n);
  const double dmean = 1.0 / (tau[0] / (wr > 1e-30 ? wr : 1e-30) + tau[1]);
  SG_CUDA(cudaMemcpyAsync(rc.scales, sc.data(), sc.size() * 8, cudaMemcpyHostToDevice, f.st));
  SG_CUDA(learn_features(f.sol, f.rhs, rc.bnext, f.w, rc.wnext, rc.diagk, f.ku, n_sk, rc.scales,
                         tau[0], tau[1], dmean, n, ld, q, rc.F1, f.st));
  rc.have_delta = false;
  if (rc.trainings > 0 && rc.r2 >= kLearnR2Min) {
    SG_TRY(mlp_forward(rc.mlp, rc.F1, n * q, rc.yhat, f.st));
    SG_CUDA(learn_to_cols(rc.yhat, n, ld, q, rc.delta, f.st));
    SG_TRY(copy_cols(f, rc.delta, rc.kin + (size_t)k * ld, q));
    rc.at_delta = k;
    k += q;
    rc.have_delta = true;
  }
  SG_TRY(copy_cols(f, f.sol, rc.xprev, q));
  // the training features stay in F0 (the captured training graph reads them there)
  SG_CUDA(cudaMemcpyAsync(rc.F0, rc.F1, (size_t)n * q * kMlpIn * sizeof(float),
                          cudaMemcpyDeviceToDevice, f.st));
  rc.have_F = true;
  SG_CUDA(cudaStreamSynchronize(f.st));
  rc.seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return Status();
}

// One AI solve Sigma x = b (one column) from a recycled start over this iteration's
// block solutions (image b_block - r_block, K-image rc.kblock), [X | U] and the previous
// solution of the same system (x on entry, K-image kx when have).  K of the new
// solution is kept in kx; have tells on return whether it was formed.
Status ai_solve_recycled(Fit& f, Recycle& rc, const double* b, double* x, double* kx, bool& have,
                         const double tau[2]) {
  const int64_t ld = f.ld;
  int mb = 0;
  rc.kv_ok = rc.have_kblock;
  SG_TRY(copy_cols(f, f.sol, rc.v, f.q));
  SG_TRY(copy_cols(f, rc.kblock, rc.kv, f.q));
  SG_CUDA(sub_cols(f.rhs, rc.br, rc.av, f.n, ld, f.q, f.st));
  mb += f.q;
  if (rc.kxu_ok || tau[1] == 0.0) {
    SG_TRY(basis_cols(f, rc, mb, f.rhs + ld, f.kxu, f.p + f.nrv, tau));
    mb += f.p + f.nrv;
    if (!rc.kxu_ok) rc.kv_ok = false;
  }
  if (rc.n_keep > 0) {  // this iteration's block directions: a Krylov basis for K P y
    SG_TRY(basis_cols(f, rc, mb, rc.keep_p, rc.keep_kp, rc.n_keep, tau));
    mb += rc.n_keep;
  }
  if (have) {
    SG_TRY(basis_cols(f, rc, mb, x, kx, 1, tau));
    mb += 1;
  }
  SG_TRY(copy_cols(f, b, rc.av + (size_t)mb * ld, 1));
  bool ok = false;
  SG_TRY(galerkin_start(f, rc, mb, 1, ok));
  bool kx_ok = false;
  if (ok) {
    SG_TRY(solve(f, b, x, rc.x0, 1, tau, rc.ax0, nullptr, kx, rc.kv_ok ? rc.kx0 : nullptr,
                 &kx_ok));
  } else {
    if (have) SG_TRY(copy_cols(f, x, rc.x0, 1));
    SG_TRY(solve(f, b, x, have ? rc.x0 : nullptr, 1, tau, nullptr, nullptr, kx, nullptr, &kx_ok));
  }
  have = kx_ok;
  return Status();
}

}  // namespace

}  // namespace saige

using namespace saige;

#define SG_API extern "C" __attribute__((visibility("default")))

SG_API void saige_ai_reml_config_default(saige_ai_reml_config* c) {
  if (!c) return;
  c->max_iter = 30;
  c->tol = 0.02;
  c->pcg_tol = 1e-5;
  c->pcg_max_iter = 500;
  c->n_random_vectors = 30;
  c->seed = 12345;
  c->precision = SAIGE_PREC_FP32;
  c->solve = SAIGE_SOLVE_SINGLE;
  c->warm_start = SAIGE_WARM_ZERO;
  c->precond = SAIGE_PRECOND_UNIT;
}

static Status fit_impl(saige_grm* h, const double* y, const double* x, int64_t n, int32_t p,
                       int32_t trait, const saige_ai_reml_config* cfg, saige_ai_reml_summary* out,
                       double* alpha_out, double* mu_out, double* eta_out, double* w_out,
                       double* tau_trace) {
  if (cfg->warm_start < SAIGE_WARM_ZERO || cfg->warm_start > SAIGE_WARM_RECYCLED)
    return fail(SAIGE_EINVAL, "unknown warm_start %d", cfg->warm_start);
  if (cfg->precond != SAIGE_PRECOND_UNIT && cfg->precond != SAIGE_PRECOND_DIAG_K)
    return fail(SAIGE_EINVAL, "unknown precond %d", cfg->precond);
  h->n_fits += 1;
  PhaseTimer tm;
  tm.launches = &h->n_kv_launches;
  tm.l0 = h->n_kv_launches;
  Fit f;
  f.h = h;
  f.st = h->stream;
  f.n = n;
  f.ld = h->n_pad;
  f.p = p;
  f.nrv = cfg->n_random_vectors;
  f.q = 1 + p + f.nrv;
  f.cfg = cfg;
  const int64_t ld = f.ld;
  // column layout of the fit workspace (each column is ld doubles)
  const size_t q = (size_t)f.q, nrv = (size_t)f.nrv, pp = (size_t)p;
  const size_t cols[] = {1, pp, 1, 1, 1, 1, 1, 1,  // y, x, eta, mu, w, wmax, d, ytil
                         q, q,                     // rhs, sol
                         pp + nrv, nrv, nrv,       // kxu, pu, tmpq
                         1, 1, 1, 1, 1, 1, 1};     // py, kpy, pk, invw_py, pw, pk_raw, pw_raw
  size_t nvec = 0;
  for (size_t c : cols) nvec += c;
  const size_t small = (size_t)(p * f.q + p * p + 4 * f.q + 64) * 8;
  const size_t part = (size_t)red_blocks(n) * (size_t)std::max(p * f.q, 3 * f.q) * 8;
  SG_TRY(f.mem.reserve(nvec * ld * 8 + small + part));
  double* base = f.mem.as<double>();
  double* const vec_end = base + nvec * ld;
  SG_CUDA(cudaMemsetAsync(base, 0, nvec * ld * 8, f.st));
  size_t ci = 0;
  auto take = [&](size_t ncol) {
    if (ci >= sizeof(cols) / sizeof(cols[0]) || cols[ci] != ncol) std::abort();
    ++ci;
    double* r = base;
    base += ncol * ld;
    return r;
  };
  f.y = take(1); f.x = take(pp); f.eta = take(1); f.mu = take(1); f.w = take(1);
  f.wmax = take(1); f.d = take(1); f.ytil = take(1);
  f.rhs = take(q); f.sol = take(q);
  f.kxu = take(pp + nrv); f.pu = take(nrv); f.tmpq = take(nrv);
  f.ku = f.kxu + pp * ld;
  f.py = take(1); f.kpy = take(1); f.pk = take(1); f.invw_py = take(1); f.pw = take(1);
  f.pk_raw = take(1); f.pw_raw = take(1);
  if (base != vec_end || ci != sizeof(cols) / sizeof(cols[0])) std::abort();
  f.dsmall = base;
  f.partial = base + small / 8;
  tm.mark("  setup");

  cudaEvent_t e0, e1;
  SG_CUDA(cudaEventCreate(&e0));
  SG_CUDA(cudaEventCreate(&e1));
  SG_CUDA(cudaEventRecord(e0, f.st));
  const int64_t kv0 = h->n_kv, kl0 = h->n_kv_launches;

  SG_CUDA(cudaMemcpyAsync(f.y, y, (size_t)n * 8, cudaMemcpyHostToDevice, f.st));
  SG_CUDA(cudaMemcpy2DAsync(f.x, (size_t)ld * 8, x, (size_t)n * 8, (size_t)n * 8, (size_t)p,
                            cudaMemcpyHostToDevice, f.st));

  // ---- GLM IRLS initialisation (ai_reml.rs:431-482) --------------------
  std::vector<double> alpha((size_t)p, 0.0), anew((size_t)p), l, xtwx((size_t)p * p),
      xtwz((size_t)p), xw;
  SG_CUDA(init_mu(f.y, trait, f.mu, f.eta, n, f.st));
  // rhs = [ytil | X] while the IRLS runs, so that X'W ytil and X'W X come from one
  // reduction (each entry's sum is the same as from two)
  SG_CUDA(cudaMemcpy2DAsync(f.rhs + ld, (size_t)ld * 8, f.x, (size_t)ld * 8, (size_t)ld * 8,
                            (size_t)p, cudaMemcpyDeviceToDevice, f.st));
  for (int it = 0; it < 25; ++it) {
    SG_CUDA(work_vectors(f.y, f.eta, f.mu, trait, f.w, f.rhs, n, f.st));
    SG_TRY(dots(f, f.x, p, f.rhs, 1 + p, f.w, xw));
    for (int j = 0; j < p; ++j) {
      xtwz[(size_t)j] = xw[(size_t)j * (1 + p)];
      for (int k = 0; k < p; ++k) xtwx[(size_t)j * p + k] = xw[(size_t)j * (1 + p) + 1 + k];
    }
    // symmetric fill as dense.rs:227-245 (j <= k computed, mirrored)
    for (int j = 0; j < p; ++j)
      for (int k = j + 1; k < p; ++k) xtwx[(size_t)k * p + j] = xtwx[(size_t)j * p + k];
    if (!cholesky(xtwx, p, l)) {
      for (int i = 0; i < p; ++i) xtwx[(size_t)i * p + i] += 1e-6;
      if (!cholesky(xtwx, p, l)) return fail(SAIGE_SINGULAR, "Matrix is not positive definite (IRLS)");
    }
    chol_solve(l, p, xtwz.data(), anew.data());
    SG_CUDA(cudaMemcpyAsync(f.dsmall, anew.data(), (size_t)p * 8, cudaMemcpyHostToDevice, f.st));
    SG_CUDA(eta_mu(f.x, p, f.dsmall, trait, f.eta, f.mu, n, ld, f.st));
    double change = 0.0;
    for (int j = 0; j < p; ++j) change += fabs(anew[(size_t)j] - alpha[(size_t)j]);
    alpha = anew;
    if (change < 1e-8) break;
  }
  SG_CUDA(cudaMemcpyAsync(f.dsmall, alpha.data(), (size_t)p * 8, cudaMemcpyHostToDevice, f.st));
  SG_CUDA(eta_mu(f.x, p, f.dsmall, trait, f.eta, f.mu, n, ld, f.st));

  // ---- probes (ai_reml.rs:121-130), fixed for the whole fit ------------
  {
    // the ChaCha8 stream is counter based: the probe matrix is generated on the GPU
    const ChaCha8 rng(cfg->seed);
    double* u = f.rhs + (size_t)(1 + p) * ld;
    SG_CUDA(rademacher_probes_dev(rng.key(), u, n, ld, f.nrv, f.st));
  }
  double* U = f.rhs + (size_t)(1 + p) * ld;
  SG_CUDA(cudaMemcpy2DAsync(f.rhs + ld, (size_t)ld * 8, f.x, (size_t)ld * 8, (size_t)ld * 8,
                            (size_t)p, cudaMemcpyDeviceToDevice, f.st));
  // K u is the same every iteration (K and the probes are fixed): one block product,
  // with K X in the same launch for the learned start (X and U are adjacent in rhs).
  // The recycled block fit forms neither: its trace takes K P u from the K-images of the
  // block solutions (K P u = K Sinv U - K Sinv X coef, both kept beside the solutions),
  // which saves the launch.
  tm.mark("  irls");
  const bool recyc = cfg->warm_start == SAIGE_WARM_RECYCLED || cfg->warm_start == SAIGE_WARM_LEARNED;
  const bool learned = cfg->warm_start == SAIGE_WARM_LEARNED && cfg->solve == SAIGE_SOLVE_BLOCK;
  const bool ku_free = recyc && !learned && cfg->solve == SAIGE_SOLVE_BLOCK;
  if (ku_free)
    SG_CUDA(cudaMemsetAsync(f.kxu, 0, (size_t)(p + f.nrv) * ld * 8, f.st));
  else if (recyc)
    SG_TRY(grm_product(h, f.rhs + ld, f.kxu, p + f.nrv, nullptr, cfg->precision, f.st));
  else
    SG_TRY(grm_product(h, U, f.ku, f.nrv, nullptr, cfg->precision, f.st));
  tm.mark("  Ku");
  // exact diag K: the DIAG_K preconditioner and a feature of the learned start (K8)
  DevBuf diagk;
  if (cfg->precond == SAIGE_PRECOND_DIAG_K || learned) {
    SG_TRY(diagk.reserve((size_t)ld * 8));
    SG_CUDA(cudaMemsetAsync(diagk.ptr, 0, (size_t)ld * 8, f.st));
    SG_TRY(grm_diag(h, diagk.as<double>(), f.st));
  }
  const double* pre_diag = cfg->precond == SAIGE_PRECOND_DIAG_K ? diagk.as<double>() : nullptr;
  Recycle rc;
  if (recyc) SG_TRY(recycle_init(f, rc, learned, diagk.as<double>(), cfg->seed));
  rc.kxu_ok = !ku_free;
  rc.with_pw = !(trait == SAIGE_TRAIT_BINARY || trait == SAIGE_TRAIT_SURVIVAL);

  const bool fix_tau_e = trait == SAIGE_TRAIT_BINARY || trait == SAIGE_TRAIT_SURVIVAL;
  double tau[2] = {1.0, 0.0};
  int converged = 0, n_iter = 0;
  const bool warm = cfg->warm_start != SAIGE_WARM_ZERO;
  double* SinvY = f.sol;
  double* SinvX = f.sol + ld;
  double* SinvU = f.sol + (size_t)(1 + p) * ld;
  DevBuf prev;
  if (warm) SG_TRY(prev.reserve((size_t)ld * f.q * 8));

  for (int iter = 0; iter < cfg->max_iter; ++iter) {
    n_iter = iter + 1;
    SG_CUDA(work_vectors(f.y, f.eta, f.mu, trait, f.w, f.ytil, n, f.st));
    SG_CUDA(sigma_diag(f.w, tau[0], tau[1], f.wmax, f.d, n, f.st, pre_diag));
    SG_CUDA(cudaMemcpyAsync(f.rhs, f.ytil, (size_t)ld * 8, cudaMemcpyDeviceToDevice, f.st));
    if (warm && f.have_prev)
      SG_CUDA(cudaMemcpyAsync(prev.ptr, f.sol, (size_t)ld * f.q * 8, cudaMemcpyDeviceToDevice, f.st));
    const double* x0 = (warm && f.have_prev) ? prev.as<double>() : nullptr;
    bool block_kx = false;
    if (recyc && cfg->solve == SAIGE_SOLVE_BLOCK) {
      SG_TRY(block_solve_recycled(f, rc, x0, tau, block_kx));
    } else if (cfg->solve == SAIGE_SOLVE_BLOCK) {
      SG_TRY(solve(f, f.rhs, f.sol, x0, f.q, tau));
    } else {
      // one solve per right-hand side, in the reference's order
      for (int c = 0; c < f.q; ++c)
        SG_TRY(solve(f, f.rhs + (size_t)c * ld, f.sol + (size_t)c * ld,
                     x0 ? x0 + (size_t)c * ld : nullptr, 1, tau));
    }
    f.have_prev = true;
    tm.mark("  block");

    // X' Sigma^-1 X and X' Sigma^-1 y (ai_reml.rs:189-205)
    // X' [Sinv y | Sinv X] in one reduction: dxy[j] = X_j . SinvY, dxs[j*p+k] = X_j . SinvX_k
    std::vector<double> dxs((size_t)p * p), dxy((size_t)p), dall;
    SG_TRY(dots(f, f.x, p, SinvY, 1 + p, nullptr, dall));
    for (int j = 0; j < p; ++j) {
      dxy[(size_t)j] = dall[(size_t)j * (1 + p)];
      for (int k = 0; k < p; ++k) dxs[(size_t)j * p + k] = dall[(size_t)j * (1 + p) + 1 + k];
    }
    std::vector<double> cmat((size_t)p * p);
    for (int j = 0; j < p; ++j)
      for (int k = j; k < p; ++k) {
        const double v = dxs[(size_t)k * p + j];  // x.col(k) . sigma_inv_x[j]
        cmat[(size_t)j * p + k] = v;
        cmat[(size_t)k * p + j] = v;
      }
    if (!cholesky(cmat, p, l)) break;  // ai_reml.rs:207-213
    chol_solve(l, p, dxy.data(), alpha.data());
    SG_CUDA(cudaMemcpyAsync(f.dsmall, alpha.data(), (size_t)p * 8, cudaMemcpyHostToDevice, f.st));
    SG_CUDA(eta_mu(f.x, p, f.dsmall, trait, f.eta, f.mu, n, ld, f.st));

    // P y = Sinv y - SinvX alpha; YPAPY = Py' K Py (ai_reml.rs:221-232)
    SG_TRY(copy_cols(f, SinvY, f.py, 1));
    SG_CUDA(sub_combo(f.py, 1, SinvX, p, f.dsmall, n, ld, f.st));
    if (recyc && cfg->solve == SAIGE_SOLVE_BLOCK && block_kx && !rc.learned) {
      SG_TRY(kpy_from_block(f, rc, alpha));  // K X*_t and K Py without a launch
    } else if (recyc && cfg->solve == SAIGE_SOLVE_BLOCK) {
      SG_TRY(kpy_recycled(f, rc, f.have_prev_pk, !fix_tau_e && f.have_prev_pw, trait, tau,
                          alpha));
    } else
      SG_TRY(grm_product(h, f.py, f.kpy, 1, nullptr, cfg->precision, f.st));
    tm.mark("  kpy");
    std::vector<double> r1;
    SG_TRY(coldots(f, f.py, f.kpy, 1, r1));
    const double ypapy = r1[0];

    // Hutchinson trace of P K (ai_reml.rs:237-258)
    SG_TRY(copy_cols(f, SinvU, f.pu, f.nrv));
    SG_TRY(p_project(f, f.pu, U, f.nrv, l));
    std::vector<double> tr;
    if (rc.kxu_ok) {
      SG_TRY(coldots(f, f.ku, f.pu, f.nrv, tr));  // (K u)' P u
    } else {
      // u' K P u with K P u = K Sinv U - K Sinv X coef (coef of the projection above,
      // still in f.dsmall; rc.kblock = K [Sinv y | Sinv X | Sinv U] of this iteration)
      SG_TRY(copy_cols(f, rc.kblock + (size_t)(1 + p) * ld, f.tmpq, f.nrv));
      SG_CUDA(sub_combo(f.tmpq, f.nrv, rc.kblock + ld, p, f.dsmall, n, ld, f.st));
      SG_TRY(coldots(f, U, f.tmpq, f.nrv, tr));
    }
    double trace_sum = 0.0;
    for (int k = 0; k < f.nrv; ++k) trace_sum += tr[(size_t)k];
    const double trace_grm = trace_sum / (double)f.nrv;
    const double score_g = ypapy - trace_grm;

    // AI = (K P y)' P (K P y) (ai_reml.rs:263-273)
    // warm start from the previous iteration's unprojected solution
    if (recyc && cfg->solve == SAIGE_SOLVE_BLOCK) {
      SG_TRY(ai_solve_recycled(f, rc, f.kpy, f.pk_raw, rc.kpk, rc.have_kpk, tau));
    } else {
      if (warm && f.have_prev_pk) SG_TRY(copy_cols(f, f.pk_raw, f.pw, 1));
      SG_TRY(solve(f, f.kpy, f.pk_raw, (warm && f.have_prev_pk) ? f.pw : nullptr, 1, tau));
    }
    f.have_prev_pk = true;
    tm.mark("  ai solve");
    SG_TRY(copy_cols(f, f.pk_raw, f.pk, 1));
    SG_TRY(p_project(f, f.pk, f.kpy, 1, l));
    SG_TRY(coldots(f, f.kpy, f.pk, 1, r1));
    const double ai_11 = r1[0];

    double score_e = 0.0, ai_00 = 0.0, ai_01 = 0.0;
    if (!fix_tau_e) {
      // trace of P W^-1 (ai_reml.rs:281-299): the probe solves repeat the ones above
      for (int k = 0; k < f.nrv; ++k)
        SG_CUDA(div_w(U + (size_t)k * ld, f.w, f.tmpq + (size_t)k * ld, n, f.st));
      SG_TRY(coldots(f, f.tmpq, f.pu, f.nrv, tr));
      double tw = 0.0;
      for (int k = 0; k < f.nrv; ++k) tw += tr[(size_t)k];
      const double trace_w = tw / (double)f.nrv;
      SG_CUDA(div_w(f.py, f.w, f.invw_py, n, f.st));
      SG_TRY(coldots(f, f.py, f.invw_py, 1, r1));
      score_e = r1[0] - trace_w;
      if (recyc && cfg->solve == SAIGE_SOLVE_BLOCK) {
        SG_TRY(ai_solve_recycled(f, rc, f.invw_py, f.pw_raw, rc.kpw, rc.have_kpw, tau));
      } else {
        if (warm && f.have_prev_pw) SG_TRY(copy_cols(f, f.pw_raw, f.tmpq, 1));
        SG_TRY(solve(f, f.invw_py, f.pw_raw, (warm && f.have_prev_pw) ? f.tmpq : nullptr, 1, tau));
      }
      f.have_prev_pw = true;
      SG_TRY(copy_cols(f, f.pw_raw, f.pw, 1));
      SG_TRY(p_project(f, f.pw, f.invw_py, 1, l));
      SG_TRY(coldots(f, f.invw_py, f.pw, 1, r1));
      ai_00 = r1[0];
      SG_TRY(coldots(f, f.invw_py, f.pk, 1, r1));
      ai_01 = r1[0];
    }

    // tau update (ai_reml.rs:329-369)
    double tn[2], max_change;
    if (fix_tau_e) {
      if (fabs(ai_11) < 1e-30) break;
      const double d1 = score_g / ai_11;
      double step = 1.0;
      double tg = tau[1] + step * d1;
      while (tg < 0.0 && step > 1e-10) {
        step *= 0.5;
        tg = tau[1] + step * d1;
      }
      tg = tg > 1e-10 ? tg : 1e-10;
      max_change = fabs(tg - tau[1]) / (fabs(tg) + fabs(tau[1]) + cfg->tol);
      tn[0] = 1.0;
      tn[1] = tg;
    } else {
      const double det = ai_00 * ai_11 - ai_01 * ai_01;
      if (fabs(det) < 1e-30) break;
      const double d0 = (ai_11 * score_e - ai_01 * score_g) / det;
      const double d1 = (-ai_01 * score_e + ai_00 * score_g) / det;
      double step = 1.0;
      double t0 = tau[0] + step * d0, t1 = tau[1] + step * d1;
      while ((t0 < 0.0 || t1 < 0.0) && step > 1e-10) {
        step *= 0.5;
        t0 = tau[0] + step * d0;
        t1 = tau[1] + step * d1;
      }
      tn[0] = t0 > 1e-10 ? t0 : 1e-10;
      tn[1] = t1 > 1e-10 ? t1 : 1e-10;
      const double c0 = fabs(tn[0] - tau[0]) / (fabs(tn[0]) + fabs(tau[0]) + cfg->tol);
      const double c1 = fabs(tn[1] - tau[1]) / (fabs(tn[1]) + fabs(tau[1]) + cfg->tol);
      max_change = c0 > c1 ? c0 : c1;
    }
    tau[0] = tn[0];
    tau[1] = tn[1];
    if (tau_trace) {
      tau_trace[2 * iter] = tau[0];
      tau_trace[2 * iter + 1] = tau[1];
    }
    if (max_change < cfg->tol) {
      converged = 1;
      break;
    }
  }

  // final W, log-likelihood (ai_reml.rs:393-414)
  SG_CUDA(work_vectors(f.y, f.eta, f.mu, trait, f.w, nullptr, n, f.st));
  SG_CUDA(cudaEventRecord(e1, f.st));
  tm.mark("  iters");
  std::vector<double> mu((size_t)n), yh(y, y + n);
  SG_CUDA(cudaMemcpyAsync(mu.data(), f.mu, (size_t)n * 8, cudaMemcpyDeviceToHost, f.st));
  if (eta_out) SG_CUDA(cudaMemcpyAsync(eta_out, f.eta, (size_t)n * 8, cudaMemcpyDeviceToHost, f.st));
  if (w_out) SG_CUDA(cudaMemcpyAsync(w_out, f.w, (size_t)n * 8, cudaMemcpyDeviceToHost, f.st));
  SG_CUDA(cudaStreamSynchronize(f.st));
  double ll = 0.0;
  if (trait == SAIGE_TRAIT_QUANTITATIVE) {
    double ss = 0.0;
    for (int64_t i = 0; i < n; ++i) ss += (yh[(size_t)i] - mu[(size_t)i]) * (yh[(size_t)i] - mu[(size_t)i]);
    ll = -0.5 * (double)n * log(2.0 * M_PI * tau[0]) - 0.5 * ss / tau[0];
  } else {
    // the terms on host threads (the logs are most of the time), summed in sample order
    // as the reference does, so the value is the same bit for bit
    std::vector<double> term((size_t)n);
    auto terms = [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i) {
        double mi = mu[(size_t)i];
        mi = mi < 1e-15 ? 1e-15 : (mi > 1.0 - 1e-15 ? 1.0 - 1e-15 : mi);
        term[(size_t)i] = yh[(size_t)i] * log(mi) + (1.0 - yh[(size_t)i]) * log(1.0 - mi);
      }
    };
    const int nt = n >= 65536 ? (int)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    std::vector<std::thread> pool;
    const int64_t per = ceil_div(n, (int64_t)nt);
    for (int t = 1; t < nt; ++t)
      pool.emplace_back(terms, std::min<int64_t>(n, t * per), std::min<int64_t>(n, (t + 1) * per));
    terms(0, std::min<int64_t>(n, per));
    for (auto& th : pool) th.join();
    for (int64_t i = 0; i < n; ++i) ll += term[(size_t)i];
  }
  tm.mark("  loglik");
  float ms = 0.f;
  SG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (mu_out) memcpy(mu_out, mu.data(), (size_t)n * 8);
  if (alpha_out) memcpy(alpha_out, alpha.data(), (size_t)p * 8);
  out->tau[0] = tau[0];
  out->tau[1] = tau[1];
  out->iterations = n_iter;
  out->converged = converged;
  out->log_likelihood = ll;
  out->n_kv = h->n_kv - kv0;
  out->n_kv_launches = h->n_kv_launches - kl0;
  out->pcg_iters = f.pcg_iters;
  out->seconds = ms * 1e-3;
  out->learned_trainings = rc.trainings;
  out->learned_uses = rc.uses;
  out->learned_r2 = rc.r2;
  out->learned_seconds = rc.seconds;
  return Status();
}

SG_API int32_t saige_fit_ai_reml(saige_grm* h, const double* y, const double* x, int64_t n,
                                 int32_t p, int32_t trait, const saige_ai_reml_config* cfg,
                                 saige_ai_reml_summary* out, double* alpha, double* mu,
                                 double* eta, double* w, double* tau_trace) {
  try {
    set_error("");
    if (!h || !y || !x || !out) return fail(SAIGE_EINVAL, "null argument").code;
    if (n != h->n) return fail(SAIGE_EINVAL, "y.len() != n_samples").code;
    if (p <= 0 || p > 64) return fail(SAIGE_EINVAL, "p must be in 1..64").code;
    if (trait < 0 || trait > 2) return fail(SAIGE_EINVAL, "unknown trait type").code;
    saige_ai_reml_config c;
    if (cfg) c = *cfg;
    else saige_ai_reml_config_default(&c);
    if (c.n_random_vectors <= 0) return fail(SAIGE_EINVAL, "n_random_vectors must be positive").code;
    if (c.max_iter < 0) return fail(SAIGE_EINVAL, "max_iter must be >= 0").code;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    DeviceGuard dg(h->device);
    if (!dg.ok) return fail(SAIGE_ECUDA, "cannot make device %d current", h->device).code;
    // the fit's work is ordered on the handle's stream
    ReleaseScope rs(ReleaseMode::kStream, h->stream);
    return fit_impl(h, y, x, n, p, trait, &c, out, alpha, mu, eta, w, tau_trace).code;
  } catch (const std::bad_alloc&) {
    return fail(SAIGE_ENOMEM, "host allocation failed").code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}

// run_loco (saige-core/src/glmm/loco.rs:54-117): one fit_ai_reml per chromosome with
// K over the markers of the other chromosomes.  The packed tiles are shared: the
// chromosome's markers are masked out between the two passes of every product and the
// product is scaled by 1/M_-c, which is the GRM the reference rebuilds from the
// remaining markers.
namespace {
struct MaskGuard {
  saige_grm* h;
  explicit MaskGuard(saige_grm* g) : h(g) {}
  ~MaskGuard() { h->masked = false; }
};
}  // namespace

SG_API int32_t saige_fit_loco(saige_grm* h, const int32_t* marker_chrom, int32_t n_chrom,
                              const double* y, const double* x, int64_t n, int32_t p,
                              int32_t trait, const saige_ai_reml_config* cfg,
                              saige_ai_reml_summary* out, double* alpha, double* mu, double* w) {
  try {
    set_error("");
    if (!h || !marker_chrom || !y || !x || !out) return fail(SAIGE_EINVAL, "null argument").code;
    if (n != h->n) return fail(SAIGE_EINVAL, "y.len() != n_samples").code;
    if (n_chrom <= 0) return fail(SAIGE_EINVAL, "n_chrom must be positive").code;
    if (p <= 0 || p > 64) return fail(SAIGE_EINVAL, "p must be in 1..64").code;
    if (trait < 0 || trait > 2) return fail(SAIGE_EINVAL, "unknown trait type").code;
    if (h->m_eff != h->m)
      return fail(SAIGE_EINVAL, "handle keeps rows outside its GRM (a streamed fit-null build)").code;
    for (int64_t j = 0; j < h->m; ++j)
      if (marker_chrom[j] < 0 || marker_chrom[j] >= n_chrom)
        return fail(SAIGE_EINVAL, "marker %lld: chromosome code %d outside 0..%d", (long long)j,
                    marker_chrom[j], n_chrom - 1).code;
    saige_ai_reml_config c;
    if (cfg) c = *cfg;
    else saige_ai_reml_config_default(&c);
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    DeviceGuard dg(h->device);
    if (!dg.ok) return fail(SAIGE_ECUDA, "cannot make device %d current", h->device).code;
    ReleaseScope rs(ReleaseMode::kStream, h->stream);
    Status s;
    {
      MaskGuard guard(h);
      s = h->excl.reserve((size_t)h->m_pad);
      std::vector<uint8_t> ex((size_t)h->m_pad, 0);
      for (int32_t k = 0; s.ok() && k < n_chrom; ++k) {
        int64_t active = 0;
        for (int64_t j = 0; j < h->m; ++j) {
          ex[(size_t)j] = marker_chrom[j] == k ? 1 : 0;
          active += ex[(size_t)j] ? 0 : 1;
        }
        // ordered on the handle's stream (which a legacy-stream copy would not be), and
        // complete before ex is rewritten for the next chromosome
        if (cudaMemcpyAsync(h->excl.ptr, ex.data(), ex.size(), cudaMemcpyHostToDevice,
                            h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess) {
          s = fail(SAIGE_ECUDA, "mask upload failed");
          break;
        }
        h->m_active = active;
        h->masked = true;
        s = fit_impl(h, y, x, n, p, trait, &c, out + k, alpha ? alpha + (int64_t)k * p : nullptr,
                     mu ? mu + (int64_t)k * n : nullptr, nullptr, w ? w + (int64_t)k * n : nullptr,
                     nullptr);
        h->masked = false;
      }
    }
    return s.code;
  } catch (const std::bad_alloc&) {
    return fail(SAIGE_ENOMEM, "host allocation failed").code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}


// Uploads the .bed into d_bed.  From pinned host memory the upload runs in marker
// chunks on a copy stream and each chunk's allele and missing counts (K1) run as soon
// as it has landed, so that the counts hide under the PCIe transfer; af, mac and
// n_valid then follow traits.rs:42-54 from the exact counts (counted = true).  From
// pageable memory it is one copy and counted = false.
static bool is_pinned(const void* p) {
  cudaPointerAttributes attr{};
  const bool pinned =
      cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  (void)cudaGetLastError();
  return pinned;
}

static Status upload_and_count(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                               const int64_t* sample_idx, int64_t n, DevBuf& d_bed,
                               std::vector<double>& af, std::vector<double>& mac,
                               std::vector<int64_t>& nv, bool& counted) {
  counted = false;
  if (!is_pinned(bed)) {
    SG_CUDA(cudaMemcpy(d_bed.ptr, bed, bed_len, cudaMemcpyHostToDevice));
    return Status();
  }
  SG_TRY(check_bed_header(bed, bed_len, n_fam, m_tot));
  std::vector<int32_t> sidx;
  bool identity = true;
  SG_TRY(check_subset(sample_idx, n, n_fam, sidx, identity));
  const int64_t bpm = (n_fam + 3) / 4;
  struct Streams {
    cudaStream_t c = nullptr, k = nullptr;
    std::vector<cudaEvent_t> ev;
    ~Streams() {
      for (cudaEvent_t e : ev) cudaEventDestroy(e);
      if (c) cudaStreamDestroy(c);
      if (k) cudaStreamDestroy(k);
    }
  } ss;
  SG_CUDA(cudaStreamCreateWithFlags(&ss.c, cudaStreamNonBlocking));
  SG_CUDA(cudaStreamCreateWithFlags(&ss.k, cudaStreamNonBlocking));
  constexpr int kChunks = 16;
  const int64_t per = ceil_div(m_tot, kChunks);
  DevBuf d_rows, d_sidx, d_cnt;
  std::vector<int64_t> rows((size_t)m_tot);
  for (int64_t j = 0; j < m_tot; ++j) rows[(size_t)j] = j;
  SG_TRY(d_rows.reserve((size_t)m_tot * 8));
  SG_TRY(d_cnt.reserve((size_t)m_tot * 2 * 8));
  SG_CUDA(cudaMemcpyAsync(d_rows.ptr, rows.data(), (size_t)m_tot * 8, cudaMemcpyHostToDevice, ss.k));
  const int32_t* sp = nullptr;
  if (!identity) {
    SG_TRY(d_sidx.reserve(sidx.size() * 4));
    SG_CUDA(cudaMemcpyAsync(d_sidx.ptr, sidx.data(), sidx.size() * 4, cudaMemcpyHostToDevice, ss.k));
    sp = d_sidx.as<int32_t>();
  }
  uint8_t* dst = d_bed.as<uint8_t>();
  for (int64_t j0 = 0; j0 < m_tot; j0 += per) {
    const int64_t j1 = std::min(m_tot, j0 + per);
    const size_t lo = j0 == 0 ? 0 : (size_t)(3 + j0 * bpm);
    const size_t hi = j1 == m_tot ? bed_len : (size_t)(3 + j1 * bpm);
    SG_CUDA(cudaMemcpyAsync(dst + lo, bed + lo, hi - lo, cudaMemcpyHostToDevice, ss.c));
    cudaEvent_t e = nullptr;
    SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ss.ev.push_back(e);
    SG_CUDA(cudaEventRecord(e, ss.c));
    SG_CUDA(cudaStreamWaitEvent(ss.k, e, 0));
    SG_CUDA(launch_bed_gather(dst, bpm, d_rows.as<int64_t>() + j0, j1 - j0, sp, n, nullptr, 0,
                              d_cnt.as<int64_t>() + 2 * j0, ss.k));
  }
  std::vector<int64_t> cnt((size_t)m_tot * 2);
  SG_CUDA(cudaMemcpyAsync(cnt.data(), d_cnt.ptr, cnt.size() * 8, cudaMemcpyDeviceToHost, ss.k));
  SG_CUDA(cudaStreamSynchronize(ss.k));
  SG_CUDA(cudaStreamSynchronize(ss.c));
  for (int64_t j = 0; j < m_tot; ++j) {
    const int64_t alt = cnt[(size_t)(2 * j)], miss = cnt[(size_t)(2 * j + 1)];
    const int64_t valid = n - miss;
    // traits.rs:42-54, the same f64 operations on the same exact integers
    const double sum = (double)alt;
    af[(size_t)j] = valid > 0 ? sum / (2.0 * (double)valid) : 0.0;
    const double other = 2.0 * (double)valid - sum;
    mac[(size_t)j] = sum < other ? sum : other;
    nv[(size_t)j] = valid;
  }
  counted = true;
  return Status();
}

SG_API int32_t saige_fit_null_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                       int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                       const double* y, const double* x, int32_t p, int32_t trait,
                                       double min_maf, double max_missing,
                                       const saige_ai_reml_config* cfg,
                                       saige_ai_reml_summary* out, double* alpha, double* mu,
                                       double* tau_trace, int64_t* m_grm_out, int64_t* m_vr_out,
                                       const saige_vr_config* vr_cfg, saige_vr_summary* vr_out) {
  try {
    set_error("");
    if (!bed || !y || !x || !out || m_tot <= 0) return fail(SAIGE_EINVAL, "null argument").code;
    saige_ai_reml_config c;
    if (cfg) c = *cfg;
    else saige_ai_reml_config_default(&c);
    if (bed_len < 3) return fail(SAIGE_EBED, "Bed file too small").code;
    PhaseTimer tm;
    // one upload of the .bed (fit_null.rs:118 maps it once as well)
    DevBuf d_bed;
    Status s = d_bed.reserve(bed_len);
    if (!s.ok()) return s.code;
    tm.mark("alloc bed");
    std::vector<double> af((size_t)m_tot), mac((size_t)m_tot);
    std::vector<int64_t> nv((size_t)m_tot);
    std::vector<int64_t> gidx, vidx;
    int64_t m_grm = 0, m_vr = 0;
    int32_t rc = SAIGE_OK;
    saige_grm* h = nullptr;
    // MIXED fits from pinned memory build the GRM while the .bed streams in
    const bool mixed_only = c.precision == SAIGE_PREC_MIXED &&
                            (!vr_out || !vr_cfg || vr_cfg->precision == SAIGE_PREC_MIXED);
    if (mixed_only && is_pinned(bed)) {
      s = stream_fit_null_grm(bed, bed_len, n_fam, m_tot, sample_idx, n, min_maf, max_missing,
                              c.seed, d_bed, af, mac, nv, vidx, m_grm, &h);
      if (!s.ok() && s.code != SAIGE_ENOMEM) return s.code;
      if (s.ok()) {
        m_vr = (int64_t)vidx.size();
        tm.mark("stream grm");
      } else {
        h = nullptr;  // short of memory for the streamed build: the steps below
        set_error("");
      }
    }
    if (!h) {
      bool counted = false;
      s = upload_and_count(bed, bed_len, n_fam, m_tot, sample_idx, n, d_bed, af, mac, nv, counted);
      if (!s.ok()) return s.code;
      tm.mark(counted ? "upload+counts" : "upload");
      if (!counted) {
        rc = saige_bed_marker_stats_dev(d_bed.as<uint8_t>(), bed_len, n_fam, m_tot, sample_idx, n,
                                        af.data(), mac.data(), nv.data());
        if (rc != SAIGE_OK) return rc;
        tm.mark("counts");
      }
      gidx.resize((size_t)m_tot);
      vidx.resize((size_t)m_tot);
      rc = saige_select_grm_markers(af.data(), mac.data(), nv.data(), m_tot, n, min_maf,
                                    max_missing, c.seed, gidx.data(), &m_grm, vidx.data(), &m_vr);
      if (rc != SAIGE_OK) return rc;
      tm.mark("select");
      std::vector<double> gaf((size_t)m_grm);
      for (int64_t j = 0; j < m_grm; ++j) gaf[(size_t)j] = af[(size_t)gidx[(size_t)j]];
      rc = saige_grm_create_from_bed_dev(d_bed.as<uint8_t>(), bed_len, n_fam, m_tot, sample_idx,
                                         n, gidx.data(), m_grm, gaf.data(), -1, &h);
      if (rc != SAIGE_OK) return rc;
      tm.mark("grm");
    }
    if (m_grm_out) *m_grm_out = m_grm;
    if (m_vr_out) *m_vr_out = m_vr;
    // the variance-ratio candidates' packed rows outlive the full .bed
    VrRows vr_rows;
    std::vector<double> vr_mac;
    if (vr_out) {
      vr_mac.resize((size_t)m_vr);
      for (int64_t j = 0; j < m_vr; ++j) vr_mac[(size_t)j] = mac[(size_t)vidx[(size_t)j]];
      Status gs = vr_gather_rows(d_bed.as<uint8_t>(), (n_fam + 3) / 4, vidx.data(), m_vr,
                                 sample_idx, n, vr_rows, h->stream);
      if (!gs.ok()) {
        saige_grm_destroy(h);
        return gs.code;
      }
    }
    d_bed.release();  // the handle holds the packed GRM rows
    tm.mark("free bed");
    std::vector<double> mu_v((size_t)n), w_v((size_t)n);
    rc = saige_fit_ai_reml(h, y, x, n, p, trait, &c, out, alpha, mu_v.data(), nullptr, w_v.data(),
                           tau_trace);
    tm.mark("fit");
    if (mu) memcpy(mu, mu_v.data(), (size_t)n * 8);
    if (rc == SAIGE_OK && vr_out) {
      saige_vr_config vc;
      if (vr_cfg) {
        vc = *vr_cfg;
      } else {
        saige_vr_config_default(&vc);
        vc.precision = c.precision;
      }
      if (m_vr == 0) {
        // fit_null.rs:352-358: no candidate, variance ratio 1
        *vr_out = saige_vr_summary{};
        vr_out->variance_ratio = 1.0;
      } else {
        std::lock_guard<std::recursive_mutex> lk(h->mu);
        cudaSetDevice(h->device);
        Status vs = vr_from_rows(h, vr_rows, vr_mac.data(), mu_v.data(), w_v.data(), out->tau,
                                 trait, x, p, &vc, vr_out);
        rc = vs.code;
      }
      tm.mark("vr");
    }
    saige_grm_destroy(h);
    tm.mark("destroy");
    return rc;
  } catch (const std::bad_alloc&) {
    return fail(SAIGE_ENOMEM, "host allocation failed").code;
  } catch (...) {
    return fail(SAIGE_EINVAL, "unexpected C++ exception").code;
  }
}
