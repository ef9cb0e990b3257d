/*
 * saige_gpu.h — C ABI of the B200 (sm_100a) fit-null GRM-product library.
 *
 * The library replaces the saige-rs fit-null hot path: the on-the-fly GRM
 * product K.v = Z (Z' v) / M computed straight from 2-bit PLINK genotypes,
 * the PCG solves of the Sigma = tau0 W^-1 + tau1 K operator, and the AI-REML
 * loop that drives them.  Every entry point below names the saige-rs
 * interface it stands in for (paths relative to the frhl/CSAIGE tree).
 *
 * Conventions
 *  - extern "C", plain pointers and sizes; no C++ exception crosses the ABI.
 *  - Every function returns an int32_t status (SAIGE_OK = 0).  On failure a
 *    message is available from saige_last_error() (thread-local).
 *  - Host-buffer entry points copy in and out; *_dev entry points take device
 *    pointers on the handle's device and run on the given stream (NULL = the
 *    handle's own stream) and return after the work is complete.
 *  - A handle owns its device memory and one CUDA stream.  Calls on one handle
 *    are serialised by an internal mutex, so concurrent callers (the rayon
 *    probe solves of ai_reml.rs:237-240) are safe.
 *  - Matrices are column-major (DenseMatrix, saige-linalg/src/dense.rs:15-39);
 *    a block of nrhs vectors of length n is n*nrhs doubles, vector-major.
 *  - There is no CPU fallback: when no sm_100 device is usable, calls that
 *    need one return SAIGE_ECUDA.
 */
#ifndef SAIGE_GPU_H
#define SAIGE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  saige-rs reports dimension mismatches by panicking
 * (assert_eq!, pcg.rs:129), PCG non-convergence as a flag, and Cholesky or
 * bed-format failures as anyhow errors; here all are codes. */
#define SAIGE_OK 0
#define SAIGE_EINVAL 1        /* bad argument / dimension mismatch          */
#define SAIGE_ENOMEM 2        /* device or host allocation failed           */
#define SAIGE_ECUDA 3         /* CUDA error or no usable sm_100 device      */
#define SAIGE_NOT_CONVERGED 4 /* iteration limit reached (results valid)    */
#define SAIGE_TIMEOUT 5       /* a bounded device wait ran out              */
#define SAIGE_SINGULAR 6      /* Cholesky / AI matrix failure               */
#define SAIGE_EBED 7          /* malformed .bed (magic, mode or size)       */
#define SAIGE_ENOTSUP 8       /* unsupported option                         */

/* Arithmetic of the GRM product.
 *  FP32:  the saige-rs arithmetic (pcg.rs:128-180): z = ((g-2p)/s) rounded to
 *         f32, v rounded to f32, f32 products and sums (CUDA cores).
 *  MIXED: v quantised per column to 24-bit fixed point, split into three
 *         int8 limbs; genotypes 0/1/2 and the missing-call indicator are exact
 *         int8 tensor-core operands (tcgen05.mma kind::i8, s32 accumulate),
 *         standardisation and limb recombination in FP64. */
#define SAIGE_PREC_FP32 0
#define SAIGE_PREC_MIXED 1

/* TraitType, saige-core/src/glmm/link.rs:7-12. */
#define SAIGE_TRAIT_BINARY 0
#define SAIGE_TRAIT_QUANTITATIVE 1
#define SAIGE_TRAIT_SURVIVAL 2

typedef struct saige_grm saige_grm;

/* Last error message of the calling thread ("" when none). */
const char* saige_last_error(void);

/* ABI version: major*10000 + minor*100 + patch. */
int32_t saige_version(void);

/* Number of usable sm_100 devices (0 when none). */
int32_t saige_device_count(void);

/* ---------------------------------------------------------------------
 * Genotype input
 * ------------------------------------------------------------------- */

/* Per-marker allele frequency, minor allele count and non-missing count
 * over the sample subset, computed integer-exact on the GPU.
 * Replaces the PlinkReader::read_marker + MarkerData::compute_af loop
 * (saige-geno/src/plink.rs:237-267, saige-geno/src/traits.rs:42-54) with the
 * bed checks of plink.rs:80-98.  bed is the whole .bed file in host memory
 * (3-byte header included); sample_idx (length n, NULL = identity) holds
 * .fam row indices in the order wanted (set_sample_subset, plink.rs:223-235).
 * af/mac/n_valid have length m_tot and are bit-identical to compute_af. */
int32_t saige_bed_marker_stats(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                               const int64_t* sample_idx, int64_t n, double* af, double* mac,
                               int64_t* n_valid);

/* Same as saige_bed_marker_stats with the .bed already in device memory. */
int32_t saige_bed_marker_stats_dev(const uint8_t* bed_dev, size_t bed_len, int64_t n_fam,
                                   int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                   double* af, double* mac, int64_t* n_valid);

/* Marker QC and the variance-ratio / GRM marker split of fit-null
 * (saige-cli/src/commands/fit_null.rs:209-259): keep af in
 * [min_maf, 1-min_maf] and missing rate <= max_missing; draw 1000 indices
 * with ChaCha8Rng::seed_from_u64(seed).gen_range(0..n_pass), sort, dedup,
 * keep MAC >= 20 for the VR pool, the rest form the GRM.  grm_idx / vr_idx
 * (capacity m_tot) receive original marker indices in increasing order.
 * Returns SAIGE_EINVAL when no marker passes QC. */
int32_t saige_select_grm_markers(const double* af, const double* mac, const int64_t* n_valid,
                                 int64_t m_tot, int64_t n, double min_maf, double max_missing,
                                 uint64_t seed, int64_t* grm_idx, int64_t* m_grm, int64_t* vr_idx,
                                 int64_t* m_vr);

/* ---------------------------------------------------------------------
 * Variance ratio (saige-core/src/glmm/variance_ratio.rs:87-246, driven as in
 * saige-cli/src/commands/fit_null.rs:290-373)
 * ------------------------------------------------------------------- */
#define SAIGE_VR_XADJUST_REFERENCE 0  /* fit_null.rs:294-306 exactly: (X'WX)^-1 X'W filled
                                         p x n row-major and read back column-major */
#define SAIGE_VR_XADJUST_PROJECTION 1 /* the projection X (X'WX)^-1 X'W g */

/* VarianceRatioConfig (variance_ratio.rs:28-56) plus the solver settings. */
typedef struct saige_vr_config {
  int32_t n_markers;       /* markers before the first CV test (30) */
  int32_t use_categorical; /* MAC-binned ratios (0) */
  double min_mac;          /* 20 */
  double ratio_cv_cutoff;  /* 0.001 */
  uint64_t seed;           /* shuffle seed (12345) */
  int32_t precision;       /* SAIGE_PREC_* of the GRM products (FP32) */
  int32_t xadjust;         /* SAIGE_VR_XADJUST_* (REFERENCE) */
  int32_t block;           /* candidates per block PCG; 0: 64 for MIXED, else n_markers then 10 */
  int32_t reserved;
} saige_vr_config;

/* VarianceRatioResult (variance_ratio.rs:59-71) plus work counters. */
typedef struct saige_vr_summary {
  double variance_ratio;
  int32_t n_markers_used;
  int32_t n_categories;    /* categorical_vr entries: (cat_upper[k], cat_vr[k]) */
  double cat_upper[8];
  double cat_vr[8];
  int32_t n_solved;        /* candidates solved (a block may solve more than are used) */
  int32_t n_blocks;
  int64_t pcg_iters;       /* PCG iterations summed over columns */
  int64_t n_kv;            /* GRM products (columns) */
  double seconds;          /* device time */
} saige_vr_summary;

int32_t saige_vr_config_default(saige_vr_config* cfg);

/* The order in which estimate_variance_ratio tries its candidates
 * (variance_ratio.rs:116-120: ChaCha8Rng::seed_from_u64(seed) and rand 0.8.5's
 * SliceRandom::shuffle of 0..n_cand).  Host only. */
int32_t saige_vr_marker_order(uint64_t seed, int64_t n_cand, int64_t* order);

/* estimate_variance_ratio(dosage_vectors, mac_values, mu, tau, trait, x,
 * xvx_inv_xv, sigma_inv, config) on the GPU: dosages are n_cand x n doubles
 * (candidate-major, NaN = missing call), mac per candidate, mu and w the fit's
 * final mean and working weights (XVX_inv_XV and Sigma^-1 are built from w and
 * tau as fit_null.rs does), x n x p column-major.  A missing call is set to
 * 2*af of the marker's called genotypes (the reference keeps NaN, which makes
 * its ratio NaN); markers without missing calls are treated as the reference
 * treats them.  per_marker_vr / used_idx (capacity n_cand, may be NULL)
 * receive the ratios and the candidate indices in the order used.  Returns
 * SAIGE_EINVAL with "No markers available ..." when no candidate is usable. */
int32_t saige_estimate_variance_ratio(saige_grm* h, const double* dosages, const double* mac,
                                      int64_t n_cand, const double* mu, const double* w,
                                      const double tau[2], int32_t trait, const double* x,
                                      int32_t p, const saige_vr_config* cfg,
                                      saige_vr_summary* out, double* per_marker_vr,
                                      int64_t* used_idx);

/* ---------------------------------------------------------------------
 * The .saige.model file (saige-core/src/model/null_model.rs:17-113,
 * serialization.rs:13-17): NullModel as bincode 1.3.3 serialises it
 * ------------------------------------------------------------------- */
/* The fields of NullModel that the caller supplies; mu2 and the residuals are
 * computed as NullModel::new does (null_model.rs:83-88).  Arrays are read only. */
typedef struct saige_null_model {
  int32_t trait;                  /* SAIGE_TRAIT_* (the TraitType variant index) */
  int32_t p;                      /* covariates including the intercept (x_ncols) */
  int64_t n;                      /* samples */
  const char* const* sample_ids;  /* n UTF-8 strings, model order */
  double tau[2];
  const double* alpha;            /* p */
  const double* mu;               /* n */
  const double* y;                /* n */
  const double* x;                /* n x p, column-major */
  const double* xvx_inv_xv;       /* p x n as fit_null.rs:294-305 fills it (data[j*n + i]) */
  double variance_ratio;          /* VarianceRatioResult */
  int32_t vr_n_categories;
  int32_t use_loco;
  const double* vr_cat_upper;     /* vr_n_categories */
  const double* vr_cat_vr;
  int64_t vr_n_markers_used;
  const double* vr_per_marker;    /* vr_n_per_marker (may be NULL: empty) */
  int64_t vr_n_per_marker;
  int32_t n_loco;                 /* per-chromosome entries (0 as fit_null writes them) */
  int32_t use_sparse_grm;
  const char* const* loco_chrom;  /* n_loco */
  const double* loco_tau;         /* 2 * n_loco */
  const double* loco_mu;          /* n_loco * n */
  const double* loco_residuals;   /* n_loco * n */
  int64_t n_markers_in_grm;       /* 0 as NullModel::new leaves it */
} saige_null_model;

/* save_model (serialization.rs:13-17): writes path (.saige.model). Host only. */
int32_t saige_write_null_model(const char* path, const saige_null_model* model);

/* XVX_inv_XV of fit_null.rs:290-305 on the host: XVX = X'WX, its inverse by
 * Cholesky unit-column solves, out[j*n + i] = sum_k inv(j,k) x(i,k) w(i)
 * (x n x p column-major, out p*n doubles). Host only. */
int32_t saige_xvx_inv_xv(const double* x, const double* w, int64_t n, int32_t p, double* out);

/* No counterpart in the reference (memory management).  Device buffers of 1 MiB
 * and more (packed genotypes, tiles, the uploaded .bed, per-marker metadata and
 * workspaces) are kept in a per-device cache when released and reused by later
 * allocations of 1 to 1.25 times their size, so that repeated fits of one cohort
 * shape skip mapping and unmapping tens of GB.  This call frees the cached blocks of
 * every device and the pinned host block of saige_fit_null_from_bed's streamed build.
 * The cache also gives its blocks back by itself when an allocation would otherwise
 * fail. */
int32_t saige_release_cached_memory(void);

/* The Rademacher probe vectors of fit_ai_reml (saige-core/src/glmm/ai_reml.rs:121-130):
 * ChaCha8Rng::seed_from_u64(seed), n_vec vectors of n entries drawn in order with
 * gen::<bool>() -> +1 / -1.  Generated on `device` (the stream is counter based)
 * and copied to out (n_vec * n doubles, vector-major). */
int32_t saige_rademacher_probes(uint64_t seed, int32_t n_vec, int64_t n, double* out,
                                int32_t device);

/* ---------------------------------------------------------------------
 * GRM operator (OnTheFlyGrm, saige-core/src/glmm/pcg.rs:91-180)
 * ------------------------------------------------------------------- */

/* OnTheFlyGrm::new (pcg.rs:101-122) from the packed bed: the markers
 * marker_idx[0..m) (rows of the .bed) over the sample subset, with the allele
 * frequencies the reference passes (grm_afs, fit_null.rs:257).  Genotypes
 * stay 2-bit packed in HBM (gathered to the subset order, padded); no dense
 * Z is materialised.  device < 0 selects the current device. */
int32_t saige_grm_create_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                  int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                  const int64_t* marker_idx, int64_t m,
                                  const double* allele_freqs, int32_t device, saige_grm** out);

/* Same as saige_grm_create_from_bed, with the .bed already in device memory
 * (bed_dev points at the 3-byte header). */
int32_t saige_grm_create_from_bed_dev(const uint8_t* bed_dev, size_t bed_len, int64_t n_fam,
                                      int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                      const int64_t* marker_idx, int64_t m,
                                      const double* allele_freqs, int32_t device,
                                      saige_grm** out);

/* OnTheFlyGrm::new with the reference's own argument (pcg.rs:101): m dosage
 * vectors of length n (marker-major, m*n doubles, NaN = missing) and their
 * allele frequencies.  Dosages must be 0, 1, 2 or NaN (hard calls). */
int32_t saige_grm_create_from_dosages(const double* dosages, int64_t n, int64_t m,
                                      const double* allele_freqs, int32_t device,
                                      saige_grm** out);

int32_t saige_grm_destroy(saige_grm* h);

/* n samples, m markers of the operator. */
int32_t saige_grm_dims(const saige_grm* h, int64_t* n, int64_t* m);

/* OnTheFlyGrm::mat_vec (pcg.rs:128-180) for nrhs vectors at once:
 * out[:,r] = K v[:,r].  v and out are n*nrhs doubles (host memory). */
int32_t saige_grm_matvec(saige_grm* h, const double* v, double* out, int64_t n, int32_t nrhs,
                         int32_t precision);

/* Device-pointer form of saige_grm_matvec. */
int32_t saige_grm_matvec_dev(saige_grm* h, const double* v_dev, double* out_dev, int64_t n,
                             int32_t nrhs, int32_t precision, void* stream);

/* The diagonal of the GRM, K_ii = (1/M) sum_m z_im^2 with z as OnTheFlyGrm::new
 * standardises it (missing -> 0), in FP64: Get_Diagof_StdGeno of SAIGE's C++
 * (src/SAIGE_fitGLMM_fast.cpp:642-680), which saige-rs does not form (its Jacobi
 * preconditioner takes K_ii = 1, ai_reml.rs:158-164).  out has n doubles. */
int32_t saige_grm_diag(saige_grm* h, double* out, int64_t n);

/* No counterpart in the reference.  FP32 product like saige_grm_matvec_dev
 * (same kernels, same results) for callers that cannot let a library call
 * cudaMalloc: processes whose own pool already holds nearly all of the GPU's
 * memory, and latency-critical callers that cannot afford the device
 * synchronisation cudaMalloc/cudaFree may cause.  It allocates nothing: its
 * scratch is a 32 MiB array compiled into the library, which every GPU that
 * loads the library holds until the process exits.  The GRM must fit in it:
 * it needs 4 n_pad (v) + 4 m_pad (u) + 4 n_splits n_pad (partial sums) bytes,
 * each part rounded up to 256, with n_pad = n rounded up to 512, m_pad = m rounded
 * up to 128 and 1 to ~6 splits, fewer as n grows (about 2.7 million samples at
 * 150,000 markers); saige_grm_noalloc_scratch_bytes gives a handle's figure.
 * Larger ones get SAIGE_EINVAL with the sizes in saige_last_error().  The first
 * call on a device (and the first after a device reset) looks up the array's
 * device address, so make that call before any stream capture.  v_dev/out_dev hold
 * nrhs columns of n doubles; the work is enqueued on `stream` (NULL: the
 * handle's stream) and the call returns without waiting for it.  All calls on
 * one device share the array: calls that overlap on the GPU race. */
int32_t saige_grm_matvec_dev_noalloc(saige_grm* h, const double* v_dev, double* out_dev,
                                     int64_t n, int32_t nrhs, void* stream);

/* No counterpart in the reference.  The static scratch that
 * saige_grm_matvec_dev_noalloc would use for this handle (need) and the size of the
 * array (limit), so that a caller can check ahead of time.  Host only. */
int32_t saige_grm_noalloc_scratch_bytes(const saige_grm* h, size_t* need, size_t* limit);

/* ---------------------------------------------------------------------
 * PCG solves
 * ------------------------------------------------------------------- */

typedef struct {
  double tol;        /* PcgSolver::tol (decomposition.rs:173-187), default 1e-5 */
  int32_t max_iter;  /* PcgSolver::max_iter, default 500                        */
  int32_t precision; /* SAIGE_PREC_*                                            */
} saige_pcg_options;

/* PcgSolver::solve (saige-linalg/src/decomposition.rs:212-298) on the
 * fit-null operator Sigma v = tau0 v / max(w,1e-30) + tau1 K v with the
 * Jacobi preconditioner 1/(tau0/max(w,1e-30) + tau1) (ai_reml.rs:142-164).
 * nrhs > 1 runs one block PCG whose columns each follow the single-vector
 * recurrence and stop on their own test ||r|| < tol*max(||b||,1).
 * x0 (nullable) is the warm start; x receives the solutions; iters, resid
 * and converged (each length nrhs, nullable) the per-column PcgResult.
 * Returns SAIGE_OK even when a column did not converge (as the reference,
 * which only sets converged = false). */
int32_t saige_pcg_solve(saige_grm* h, const double* w, const double tau[2], const double* b,
                        const double* x0, double* x, int64_t n, int32_t nrhs,
                        const saige_pcg_options* opt, int32_t* iters, double* resid,
                        uint8_t* converged);

/* solve_mixed_model_pcg (saige-core/src/glmm/pcg.rs:37-78): the score-test
 * convention Sigma v = tau0 w v + tau1 K v with preconditioner
 * 1/(tau0 w + tau1) (unchanged when |diag| <= 1e-30), single vector. */
int32_t saige_solve_mixed_model_pcg(saige_grm* h, const double tau[2], const double* w,
                                    const double* b, double* x, int64_t n,
                                    const saige_pcg_options* opt, int32_t* iters, double* resid,
                                    uint8_t* converged);

/* ---------------------------------------------------------------------
 * AI-REML (fit_ai_reml, saige-core/src/glmm/ai_reml.rs:86-427)
 * ------------------------------------------------------------------- */

/* Solve strategies beyond the reference's (the reference is
 * SAIGE_SOLVE_SINGLE with SAIGE_WARM_ZERO). */
#define SAIGE_SOLVE_SINGLE 0 /* one PCG per right-hand side, as ai_reml.rs     */
#define SAIGE_SOLVE_BLOCK 1  /* y, X columns and probes in one block PCG        */

#define SAIGE_WARM_ZERO 0     /* x0 = 0 (the reference)                        */
#define SAIGE_WARM_PREVIOUS 1 /* previous AI-REML iteration's solution         */
/* Jacobi preconditioner of the fit-null PCG.  UNIT: 1 / (tau0 / w + tau1), the
 * saige-rs form that takes diag K = 1 (ai_reml.rs:142-164); DIAG_K: 1 / (tau0 / w +
 * tau1 K_ii) with the exact diagonal, as SAIGE's C++ does (SAIGE_fitGLMM_fast.cpp:
 * 2037-2080, Get_Diagof_StdGeno :642-680). */
#define SAIGE_PRECOND_UNIT 0
#define SAIGE_PRECOND_DIAG_K 1

#define SAIGE_WARM_LEARNED 2  /* recycled start plus a learned correction (MLP
                                 trained on the fit's own solves), used when it
                                 validates; the recycled start otherwise        */
#define SAIGE_WARM_RECYCLED 3 /* Galerkin start over vectors whose Sigma-image
                                 needs no GRM product: X, the probes, the
                                 previous solutions (block solve only)          */

typedef struct {
  int32_t max_iter;         /* AiRemlConfig::max_iter (ai_reml.rs:22-51), 30     */
  double tol;               /* tau tolerance, 0.02 (fit-null CLI passes --tol)   */
  double pcg_tol;           /* 1e-5                                              */
  int32_t pcg_max_iter;     /* 500                                               */
  int32_t n_random_vectors; /* 30                                                */
  uint64_t seed;            /* 12345                                             */
  int32_t precision;        /* SAIGE_PREC_*                                      */
  int32_t solve;            /* SAIGE_SOLVE_*                                     */
  int32_t warm_start;       /* SAIGE_WARM_*                                      */
  int32_t precond;          /* SAIGE_PRECOND_*                                   */
} saige_ai_reml_config;

typedef struct {
  double tau[2];
  int32_t iterations;
  int32_t converged;
  double log_likelihood;
  int64_t n_kv;            /* GRM products (columns) performed               */
  int64_t n_kv_launches;   /* GRM product launches (a block counts once)     */
  int64_t pcg_iters;       /* sum over solves of PCG iterations              */
  double seconds;          /* device wall time of the fit                    */
  int32_t learned_trainings; /* SAIGE_WARM_LEARNED: training rounds of the MLP  */
  int32_t learned_uses;      /* block solves whose start used its prediction   */
  double learned_r2;         /* held-out R^2 of the last training round        */
  double learned_seconds;    /* time spent on features, training, inference    */
} saige_ai_reml_summary;

/* Fill cfg with AiRemlConfig::default() (ai_reml.rs:39-51) and the
 * reference's solve strategy. */
void saige_ai_reml_config_default(saige_ai_reml_config* cfg);

/* fit_ai_reml: y (n), x (n x p column-major, intercept included), trait
 * SAIGE_TRAIT_*.  alpha (p), mu/eta/w (n) and tau_trace (2*max_iter: tau
 * after each iteration) are optional outputs.  Returns SAIGE_SINGULAR when
 * the initial IRLS Cholesky fails (the reference's only error path);
 * non-convergence is reported in out->converged. */
int32_t saige_fit_ai_reml(saige_grm* h, const double* y, const double* x, int64_t n, int32_t p,
                          int32_t trait, const saige_ai_reml_config* cfg,
                          saige_ai_reml_summary* out, double* alpha, double* mu, double* eta,
                          double* w, double* tau_trace);

/* run_loco (saige-core/src/glmm/loco.rs:54-117): for each chromosome code k in
 * 0..n_chrom-1, fit_ai_reml with the GRM over the handle's markers whose
 * marker_chrom (one code per GRM marker) differs from k.  The handle's packed
 * genotypes are shared; the chromosome's markers are left out of every product
 * and the product is scaled by 1/M_-k.  out has n_chrom entries; alpha (n_chrom*p),
 * mu and w (n_chrom*n) are optional.  The reference visits chromosomes in sorted
 * name order: give codes in that order. */
int32_t saige_fit_loco(saige_grm* h, const int32_t* marker_chrom, int32_t n_chrom,
                       const double* y, const double* x, int64_t n, int32_t p, int32_t trait,
                       const saige_ai_reml_config* cfg, saige_ai_reml_summary* out,
                       double* alpha, double* mu, double* w);

/* The fit-null pipeline of saige-cli/src/commands/fit_null.rs:199-287 from
 * host buffers in one call: marker statistics over the sample subset
 * (plink.rs:237-267), QC and the VR/GRM split (fit_null.rs:209-259), the GRM
 * operator over the GRM markers (pcg.rs:101-122) and fit_ai_reml
 * (ai_reml.rs:86-427).  The .bed is copied to the device once.  Phenotype
 * and covariate parsing stay with the caller (y, x as for saige_fit_ai_reml).
 * m_grm / m_vr (optional) receive the marker split sizes.  When vr_out is not
 * NULL the variance ratio over the VR candidates follows the fit as in
 * fit_null.rs:290-373 (vr_cfg NULL: defaults with the fit's precision; no
 * candidate gives a ratio of 1). */
int32_t saige_fit_null_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                                const int64_t* sample_idx, int64_t n, const double* y,
                                const double* x, int32_t p, int32_t trait, double min_maf,
                                double max_missing, const saige_ai_reml_config* cfg,
                                saige_ai_reml_summary* out, double* alpha, double* mu,
                                double* tau_trace, int64_t* m_grm, int64_t* m_vr,
                                const saige_vr_config* vr_cfg, saige_vr_summary* vr_out);

/* ---------------------------------------------------------------------
 * Instrumentation (the reference logs per-phase times through `tracing`,
 * saige-cli/src/main.rs:53-65; here the GPU kernels are timed with CUDA
 * events on the handle's stream)
 * ------------------------------------------------------------------- */
typedef struct {
  int64_t n_kv;               /* GRM product columns                         */
  int64_t n_kv_launches;      /* GRM product calls                           */
  int64_t tc_pass_a_launches; /* tensor-core product, pass u = Z'v           */
  int64_t tc_pass_b_launches; /* tensor-core product, pass y = Z u / M       */
  double tc_pass_a_ms;        /* summed device time (profiling on)           */
  double tc_pass_b_ms;
  int64_t fp32_launches;      /* FP32 product columns                        */
  double fp32_ms;
  int64_t sc_launches;        /* MIXED single-column products on the CUDA    */
  double sc_ms;               /* cores (both passes; dp4a, same sums)        */
  int64_t sc_list_launches;   /* of those, with the missing-call lists: sums */
                              /* over the missing calls in place of dense    */
                              /* flag sums, the same integers; built at the  */
                              /* first such product of the handle's second   */
                              /* fit (env SAIGE_SR_LISTS=2: its first        */
                              /* product, =0: never)                         */
  int64_t missing_listed;     /* missing calls in the handle's lists; -1     */
                              /* while none are built or when declined       */
                              /* (over 3 % of the calls missing, or too      */
                              /* little free device memory)                  */
} saige_grm_stats;

/* Turn per-kernel CUDA-event timing on (1) or off (0) for a handle. */
int32_t saige_grm_set_profiling(saige_grm* h, int32_t on);
int32_t saige_grm_get_stats(const saige_grm* h, saige_grm_stats* out);
int32_t saige_grm_reset_stats(saige_grm* h);

/* Kernels this library has launched in the process so far. */
int64_t saige_kernel_launches(void);

/* Timed candidate launches of the tensor-core ring-shape autotuner in this process.
 * The first MIXED products of each (pass, column group, size class) of at least ~4 GB
 * of code tiles each run with the next candidate ring shape, timed with CUDA events; once
 * every candidate has run, the fastest is kept.  The candidates are real products —
 * results are identical for all shapes — so tuning adds no launches.
 * SAIGE_TC_AUTOTUNE=0 in the environment keeps the fixed shape, =2 tunes every size. */
int64_t saige_tc_autotune_trials(void);

/* No counterpart in the reference (fault handling).  Every wait of the tensor-core
 * product's pipeline (on its copies and on its MMAs) is bounded; when one runs out,
 * the kernel stops issuing work, lets what it already issued complete, frees its
 * tensor memory and returns, and the call reports SAIGE_TIMEOUT; the handle and the
 * context stay usable.  This sets the bound in SM cycles for the whole process:
 * cycles < 0 restores the default (~2 s), 0 makes every wait that is not already
 * satisfied give up at once (how the timeout path is tested). */
int32_t saige_tc_set_wait_budget(int64_t cycles);

/* ---------------------------------------------------------------------
 * Explicit GRM: replaces compute_dense_grm (saige-core/src/grm/dense.rs:22-112),
 * compute_grm_from_dosages (dense.rs:115-186), compute_sparse_grm
 * (grm/sparse.rs:18-66), compute_sparse_grm_from_dosages (sparse.rs:69-98) and
 * write_sparse_grm (saige-geno/src/sparse_grm_io.rs:73-115), the steps of the
 * create-sparse-grm command (saige-cli/src/commands/create_sparse_grm.rs:37-71).
 *
 * K_ij = (1/M) sum over the M used markers of z_i z_j, each entry one f64 sum in
 * marker order.  SAIGE_GRM_ARITH_REFERENCE rounds each product and each sum as
 * the reference does, so K is bit-identical to it; SAIGE_GRM_ARITH_FMA fuses them
 * (twice the FP64 rate, last-bit differences).
 * ------------------------------------------------------------------- */
#define SAIGE_GRM_ARITH_REFERENCE 0
#define SAIGE_GRM_ARITH_FMA 1

typedef struct {
  double min_maf;            /* .bed entry points: markers with af < min_maf or
                                af > 1 - min_maf are skipped (dense.rs:37-39)      */
  double relatedness_cutoff; /* sparse: keep i == j or |K_ij| >= cutoff            */
  int32_t arith;             /* SAIGE_GRM_ARITH_*                                  */
  int32_t device;            /* CUDA device, -1 = current                          */
  int32_t reserved[4];
} saige_explicit_grm_config;

typedef struct {
  int64_t n_markers_used;    /* M (the usize dense.rs:22 returns)                  */
  int64_t nnz;               /* sparse: stored entries (upper triangle with the
                                diagonal); dense: n * n                            */
  double kernel_seconds;     /* the GRM kernel, CUDA events on the call's stream   */
  double total_seconds;      /* the whole call, host copies included               */
  double terms;              /* n (n + 1) / 2 * M products summed                  */
} saige_explicit_grm_info;

/* Sparse GRM result: the upper triangle with the diagonal, sorted by row then
 * column (the entries write_sparse_grm lists). */
typedef struct saige_sparse_grm saige_sparse_grm;

/* min_maf 0.01, relatedness_cutoff 0.125 (the command's defaults), reference
 * arithmetic, current device. */
int32_t saige_explicit_grm_config_default(saige_explicit_grm_config* cfg);

/* compute_dense_grm on a PLINK .bed (3-byte header + m_tot rows of ceil(n_fam/4)
 * bytes) over all n_fam samples (sample_idx NULL, n = n_fam) or sample_idx[0..n).
 * af as MarkerData::compute_af (saige-geno/src/traits.rs:42-54).  out: n x n
 * (symmetric: row- and column-major agree).  All zeros when no marker is used. */
int32_t saige_dense_grm_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                 int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                 const saige_explicit_grm_config* cfg, double* out,
                                 saige_explicit_grm_info* info);

/* compute_sparse_grm: the same K thresholded (sparse.rs:36-53).  *out is freed
 * with saige_sparse_grm_free. */
int32_t saige_sparse_grm_from_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam,
                                  int64_t m_tot, const int64_t* sample_idx, int64_t n,
                                  const saige_explicit_grm_config* cfg, saige_sparse_grm** out,
                                  saige_explicit_grm_info* info);

/* compute_grm_from_dosages: dosages m x n (row j = marker j, NaN = missing), af[m]
 * as given; markers with 2 af (1 - af) < 1e-10 are skipped; min_maf is not used.
 * m == 0 is the 0 x 0 matrix (out not written). */
int32_t saige_grm_from_dosages(const double* dosages, const double* af, int64_t n, int64_t m,
                               const saige_explicit_grm_config* cfg, double* out,
                               saige_explicit_grm_info* info);

/* compute_sparse_grm_from_dosages. */
int32_t saige_sparse_grm_from_dosages(const double* dosages, const double* af, int64_t n,
                                      int64_t m, const saige_explicit_grm_config* cfg,
                                      saige_sparse_grm** out, saige_explicit_grm_info* info);

int64_t saige_sparse_grm_n(const saige_sparse_grm* g);
int64_t saige_sparse_grm_nnz(const saige_sparse_grm* g);
int64_t saige_sparse_grm_n_markers(const saige_sparse_grm* g);
/* Copies the nnz entries (0-based rows and columns). */
int32_t saige_sparse_grm_get(const saige_sparse_grm* g, int32_t* rows, int32_t* cols,
                             double* vals);
void saige_sparse_grm_free(saige_sparse_grm* g);
/* A sparse GRM from upper-triangle entries sorted by row, then column (0-based),
 * e.g. to write one read back from a file.  No reference counterpart. */
int32_t saige_sparse_grm_from_triplets(int64_t n, int64_t nnz, const int32_t* rows,
                                       const int32_t* cols, const double* vals,
                                       int64_t n_markers_used, saige_sparse_grm** out);

/* write_sparse_grm: sample IDs one per line to ids_path, then the MatrixMarket
 * "coordinate real symmetric" header, "n n nnz" and 1-based "i j value" lines
 * with ten decimals to mtx_path. */
int32_t saige_write_sparse_grm(const saige_sparse_grm* g, const char* const* sample_ids,
                               int64_t n_ids, const char* mtx_path, const char* ids_path);

/* Fit-null of n_cohorts sub-cohorts of one .bed (sample_idx[c][0..n[c]), y[c],
 * x[c] n[c] x p column-major): per cohort the steps of saige_fit_null_from_bed
 * without the variance ratio (counts, QC and VR/GRM split over the cohort's samples,
 * GRM, AI-REML) — fit_null::run per cohort (fit_null.rs:199-287).  The .bed is
 * uploaded once.  With concurrent != 0 the .bed streams in by marker chunks while one
 * launch per chunk counts every cohort's alleles and missing calls and (MIXED fits)
 * one more gathers the chunk's QC-passing markers into every cohort's GRM (pinned host
 * memory lets both run under the transfer; FP32 fits gather in one pass after it), and
 * the fits run on a pool of host threads, each cohort on its own stream; the results
 * are bit-identical to the sequential ones (concurrent == 0).  Rows of more than
 * 200 KB (over 800,000 samples) take the per-cohort steps on the threads instead.  out[c], alpha[c] (p, may be
 * NULL), m_grm[c] (may be NULL); wall_seconds (may be NULL) = the whole call. */
int32_t saige_fit_null_cohorts(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                               int32_t n_cohorts, const int64_t* const* sample_idx,
                               const int64_t* n, const double* const* y, const double* const* x,
                               int32_t p, int32_t trait, double min_maf, double max_missing,
                               const saige_ai_reml_config* cfg, int32_t concurrent,
                               saige_ai_reml_summary* out, double* const* alpha, int64_t* m_grm,
                               double* wall_seconds);

/* ---------------------------------------------------------------------
 * The MLP of the learned PCG start (SAIGE_WARM_LEARNED; no reference
 * counterpart).  16 inputs, three tanh layers of 256, a linear output; BF16
 * weights and activations in the forward pass (the two 256 x 256 layers on the
 * tensor cores), FP32 arithmetic and FP32 master weights.
 * Parameter layout: W1[256][16], b1[256], W2[256][256], b2[256], W3[256][256],
 * b3[256], w4[256], b4.  These entry points expose the network's own kernels so
 * that they can be checked against a CPU reference.
 * ------------------------------------------------------------------- */
int32_t saige_mlp_param_count(void);
/* The initial weights the fit uses for a seed (uniform +-1/sqrt(fan_in)). */
int32_t saige_mlp_initial_params(uint64_t seed, float* params);
/* n_ex examples of 16 features (row-major): out[e] = MLP(features[e]) (may be NULL);
 * grad (may be NULL) = gradient of mean_e (out[e] - targets[e])^2 with respect to
 * params (through the BF16 roundings); sse (may be NULL) = sum_e (out[e] - targets[e])^2. */
int32_t saige_mlp_eval(const float* params, const float* features, const float* targets,
                       int64_t n_ex, float* out, float* grad, double* sse, int32_t device);
/* Trains params in place with the fit's trainer: steps Adam steps (lr) on
 * mini-batches of 8192 examples from e = c * n + i (q columns of n samples),
 * samples i % holdout == 0 held out; held-out mean squared error before and after
 * and the held-out mean squared target. */
int32_t saige_mlp_train(float* params, const float* features, const float* targets, int64_t n,
                        int32_t q, int32_t steps, float lr, int32_t holdout,
                        double* val_mse_before, double* val_mse_after, double* val_target_ms,
                        int32_t device);

/* ---------------------------------------------------------------------
 * Synthetic cohorts (seeded; no counterpart in the reference — test and
 * benchmark input).  Deterministic functions of the spec: the host and the
 * device generator produce identical bytes.
 * ------------------------------------------------------------------- */
typedef struct {
  uint64_t seed;
  int64_t n;            /* samples                                            */
  int64_t m;            /* markers                                            */
  double sib_frac;      /* fraction of samples in sibling pairs               */
  double cousin_frac;   /* fraction of samples in first-cousin pairs          */
  double missing_rate;  /* MCAR missing-call rate                             */
  double maf_lo, maf_hi;/* allele frequency ~ U(maf_lo, maf_hi)               */
  int32_t trait;        /* SAIGE_TRAIT_BINARY or SAIGE_TRAIT_QUANTITATIVE     */
  int32_t n_covar;      /* covariates (intercept not counted)                 */
  double prevalence;    /* binary: target case fraction                       */
  double h2;            /* heritability of the polygenic score                */
  int32_t n_causal;     /* causal markers for the polygenic score             */
  int32_t reserved;
} saige_cohort_spec;

/* Writes the .bed bytes (3-byte header + m * ceil(n/4)) into bed_out, which
 * is device memory when on_device != 0. */
int32_t saige_gen_bed(const saige_cohort_spec* spec, uint8_t* bed_out, int32_t on_device);

/* Phenotype y (n) and design x (n x (1+n_covar), column-major, column 0 the
 * intercept). */
int32_t saige_gen_pheno(const saige_cohort_spec* spec, double* y, double* x);

#ifdef __cplusplus
}
#endif
#endif /* SAIGE_GPU_H */
