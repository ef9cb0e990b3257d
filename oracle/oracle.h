/*
 * CPU oracle for the saige-rs fit-null GRM-product path — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference algorithm, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
 * The product library (csaige_b200) never links, loads or calls it.
 *
 * Every function cites the saige-rs file:line it restates (paths relative to
 * the frhl/CSAIGE tree).  Parity pins: the 2-bit decode known answers
 * (saige-geno/src/plink.rs:288-303), PLINK's own .frq MAF column for the
 * extdata/input/plinkforGRM_1000samples_10kMarkers fixture, the PCG
 * known-answer tests (saige-linalg/src/decomposition.rs:469-526,
 * saige-core/src/glmm/pcg.rs:202-222), the Cholesky tests
 * (decomposition.rs:371-407) and the ChaCha block function against an
 * independent ChaCha20 implementation.  The ChaCha8/PCG32/rand mapping
 * streams themselves (rand 0.8.5, rand_chacha 0.3.1, rand_core 0.6.4) have no
 * golden vector in the reference: that boundary is "parity unpinned".
 */
#ifndef SAIGE_ORACLE_H
#define SAIGE_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- PLINK .bed decode and per-marker counts ------------------------- */
double orc_decode_genotype(uint8_t byte, int offset);
void orc_read_marker(const uint8_t* bed, int64_t bytes_per_marker, int64_t n_fam, int64_t marker,
                     const int64_t* sample_idx, int64_t n, double* dosages_out);
void orc_compute_af(const double* dosages, int64_t n, double* af, double* mac, int64_t* n_valid);
int orc_marker_stats(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                     const int64_t* sample_idx, int64_t n, double* af, double* mac,
                     int64_t* n_valid);

/* ---- rand 0.8.5 / rand_chacha 0.3.1 restatement ----------------------- */
typedef struct {
  uint32_t key[8];
  uint64_t counter; /* next block counter */
  uint64_t stream;
  uint32_t buf[64]; /* 4 blocks */
  int idx;          /* next word in buf; 64 = empty */
  int rounds;
} orc_chacha_rng;

void orc_chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds,
                      uint32_t out[16]);
void orc_chacha_seed_from_u64(orc_chacha_rng* r, uint64_t seed, int rounds);
void orc_chacha_from_seed(orc_chacha_rng* r, const uint8_t seed[32], int rounds);
uint32_t orc_rng_next_u32(orc_chacha_rng* r);
uint64_t orc_rng_next_u64(orc_chacha_rng* r);
int orc_rng_gen_bool(orc_chacha_rng* r);
uint64_t orc_rng_gen_range_u64(orc_chacha_rng* r, uint64_t low, uint64_t high);
void orc_rademacher_probes(uint64_t seed, int n_vec, int64_t n, double* out);

/* ---- marker QC and the VR/GRM split (fit_null.rs:209-259) ------------- */
int orc_select_markers(const double* af, const double* mac, const int64_t* n_valid, int64_t m_tot,
                       int64_t n, double min_maf, double max_missing, uint64_t seed,
                       int64_t* grm_idx, int64_t* m_grm, int64_t* vr_idx, int64_t* m_vr,
                       int64_t* n_pass);

/* ---- on-the-fly GRM (pcg.rs:91-180) ----------------------------------- */
/* mode 0: FP64 z and FP64 sums.  mode 1: saige-rs f32 z, f32 sums in the
 * sequential order a single rayon thread produces. */
void orc_grm_standardize(const double* dosages, const double* af, int64_t n, int64_t m, int mode,
                         double* z_out);
void orc_grm_matvec(const double* z, int64_t n, int64_t m, const double* v, double* out, int mode);
void orc_grm_explicit(const double* z, int64_t n, int64_t m, double* k_out);
/* pcg.rs:128-180 arithmetic (f32 z from pcg.rs:101-122, f32 dot and axpy per
 * marker, one f32 accumulator per thread, summed at the end as rayon's
 * fold/reduce does) on packed PLINK rows: markers rows[0..m) of the .bed
 * body (bed points past the 3-byte header), all n_fam samples in order.
 * threads <= 0 uses every OpenMP thread.  Returns the threads used. */
/* The product K V = Z (Z' V) / M of pcg.rs:101-180 in FP64 (its own summation order)
 * (z = (g - 2p)/sqrt(2p(1-p)) in f64, missing -> 0, zero rows when the denominator is
 * <= 1e-10) on packed rows, nrhs columns of n (column-major) at once, all threads:
 * the FP64 reference for the accuracy of the GPU products at sizes where an explicit
 * Z does not fit in host memory.  Returns the threads used. */
int orc_grm_matmul_f64_packed(const uint8_t* bed_body, int64_t bytes_per_marker, int64_t n,
                              const int64_t* rows, int64_t m, const double* af, const double* v,
                              int nrhs, double* out);
int orc_grm_matvec_f32_packed(const uint8_t* bed_body, int64_t bytes_per_marker, int64_t n,
                              const int64_t* rows, int64_t m, const double* af, const double* v,
                              double* out, int threads);

/* ---- linear algebra (decomposition.rs:35-89, 212-298) ------------------ */
int orc_cholesky(const double* a, int p, double* l);
void orc_chol_solve(const double* l, int p, const double* b, double* x);
int orc_pcg_dense(const double* a, int n, const double* b, double tol, int max_iter, double* x,
                  int* iters, double* resid);

/* ---- link / family (link.rs:29-100, family.rs:23-90) ------------------- */
enum { ORC_BINARY = 0, ORC_QUANTITATIVE = 1, ORC_SURVIVAL = 2 };
double orc_link(int trait_type, double mu);
double orc_inv_link(int trait_type, double eta);
double orc_update_mu(int trait_type, double eta);
double orc_working_weight(int trait_type, double mu);
double orc_initialize_mu(int trait_type, double y);

/* ---- GLM IRLS and AI-REML (ai_reml.rs:86-482) ------------------------- */
int orc_fit_glm_irls(const double* y, const double* x, int64_t n, int p, int trait_type,
                     int max_iter, double* alpha);

typedef struct {
  int max_iter;
  double tol;
  double pcg_tol;
  int pcg_max_iter;
  int n_random_vectors;
  uint64_t seed;
} orc_ai_reml_config;

typedef struct {
  double tau[2];
  int iterations;
  int converged;
  double log_likelihood;
  int64_t n_kv;        /* GRM products performed */
  int64_t pcg_iters;   /* total PCG iterations */
} orc_ai_reml_summary;

/* GRM operator kinds for the AI-REML oracle. */
enum { ORC_K_IDENTITY = 0, ORC_K_OTF = 1, ORC_K_EXPLICIT = 2 };

/* grm: for ORC_K_OTF the standardized z (m x n, marker-major) with kmode 0 (FP64),
 * 1 (saige-rs f32 arithmetic, one thread) or 2 (saige-rs f32 arithmetic on all host
 * threads: the rayon fold and reduce of pcg.rs:149-176);
 * for ORC_K_EXPLICIT the dense n x n K (row-major).  tau_trace (optional,
 * length 2*max_iter) receives tau after each iteration.  alpha/mu/eta/w
 * (optional) receive the final state. */
int orc_fit_ai_reml(const double* y, const double* x, int64_t n, int p, int trait_type,
                    int kind, const double* grm, int64_t m, int kmode,
                    const orc_ai_reml_config* cfg, orc_ai_reml_summary* out, double* tau_trace,
                    double* alpha, double* mu, double* eta, double* w);

/* Sigma-operator PCG for one right-hand side, the form fit_ai_reml uses
 * (ai_reml.rs:142-175): Sigma v = tau0 v / max(w,1e-30) + tau1 K v. */
int orc_pcg_sigma(const double* y_unused, int kind, const double* grm, int64_t n, int64_t m,
                  int kmode, const double* w, const double tau[2], const double* b,
                  const double* x0, double tol, int max_iter, double* x, int* iters,
                  double* resid, int* converged);

/* rand 0.8.5 UniformInt<u32>::sample_single(low, high): 32-bit widening multiply. */
uint32_t orc_rng_gen_range_u32(orc_chacha_rng* r, uint32_t low, uint32_t high);

/* variance_ratio.rs:116-120: indices 0..len shuffled by rand 0.8.5's
 * SliceRandom::shuffle with ChaCha8Rng::seed_from_u64(seed). */
void orc_shuffled_indices(uint64_t seed, int64_t len, int64_t* out);

/* Variance ratio (variance_ratio.rs:87-246 driven as in fit_null.rs:290-373).
 * dosages: n_cand x n (candidate-major), NaN = missing call; mac per candidate.
 * mu, w: the fit's final mu and working weights; x: n x p column-major.
 * xadjust 0 = as fit_null.rs:294-306 builds XVX_inv_XV (a p x n row-major array
 * read back as column-major), 1 = the projection X (X'WX)^-1 X'W g.
 * Missing calls are set to 2*af of the called genotypes (saige-rs keeps NaN,
 * which makes its variance ratio NaN).  per_marker_vr / used_idx (capacity
 * n_cand) receive the ratios and candidate indices in the order used.
 * Returns 0, or 1 when no marker is usable ("No markers available ..."). */
typedef struct {
  int n_markers;
  double min_mac;
  double ratio_cv_cutoff;
  uint64_t seed;
  int use_categorical;
  int xadjust;
} orc_vr_config;

typedef struct {
  double variance_ratio;
  int n_markers_used;
  int n_categories;
  double cat_upper[8];
  double cat_vr[8];
  int64_t n_kv;
} orc_vr_summary;

int orc_variance_ratio(const double* dosages, const double* mac, int64_t n_cand, const double* mu,
                       const double* w, const double tau[2], int trait_type, const double* x,
                       int64_t n, int p, int kind, const double* grm, int64_t m, int kmode,
                       const orc_vr_config* cfg, orc_vr_summary* out, double* per_marker_vr,
                       int64_t* used_idx);

/* ---- explicit GRM (saige-core/src/grm/dense.rs, grm/sparse.rs) -------- */
/* compute_dense_grm (dense.rs:22-112): markers of the .bed (all n_fam
 * samples, or sample_idx[0..n)) whose af (traits.rs:42-54) is within
 * [min_maf, 1 - min_maf] and whose 2 af (1 - af) is at least 1e-10, z =
 * (d - 2 af) / sqrt(2 af (1 - af)) with a missing call at the mean (z = 0),
 * K_ij = (sum over markers in file order of z_i * z_j, f64 multiply then add)
 * * (1 / n_used); all zeros when no marker is used.  out: n x n. */
int orc_dense_grm_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                      const int64_t* sample_idx, int64_t n, double min_maf, double* out,
                      int64_t* n_used);
/* compute_grm_from_dosages (dense.rs:115-186): dosages m x n (row per marker,
 * NaN = missing), af as given, only the 2 af (1 - af) < 1e-10 skip. */
void orc_grm_from_dosages(const double* dosages, const double* af, int64_t n, int64_t m,
                          double* out, int64_t* n_used);

/* ---------------------------------------------------------------------
 * The seeded synthetic cohort of the tests and the benchmark (no reference
 * counterpart), restated from the library's generator so that the CPU arm of the
 * benchmark needs nothing from the library; the tests check both byte for byte.
 * Same fields and layout as saige_cohort_spec.
 * ------------------------------------------------------------------- */
typedef struct {
  uint64_t seed;
  int64_t n, m;
  double sib_frac, cousin_frac, missing_rate, maf_lo, maf_hi;
  int32_t trait, n_covar;
  double prevalence, h2;
  int32_t n_causal, reserved;
} orc_cohort_spec;

/* .bed bytes (3-byte header + m * ceil(n/4)), all host threads. */
void orc_gen_bed(const orc_cohort_spec* spec, uint8_t* bed_out);
/* y (n) and x (n x (1 + n_covar), column-major, intercept first). */
void orc_gen_pheno(const orc_cohort_spec* spec, double* y, double* x);

#ifdef __cplusplus
}
#endif
#endif
