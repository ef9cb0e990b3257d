/*
 * CPU oracle for the saige-rs fit-null GRM-product path — TEST INFRASTRUCTURE ONLY.
 * See oracle.h for what pins it.  Built with -ffp-contract=off so that no
 * multiply-add is fused, which is what rustc emits for the reference.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ===================================================================== */
/* PLINK .bed decode                                                      */
/* ===================================================================== */

/* saige-geno/src/plink.rs:170-179: 2-bit code, low bits first;
 * 00 -> 2 (hom A1), 01 -> missing, 10 -> 1 (het), 11 -> 0 (hom A2). */
double orc_decode_genotype(uint8_t byte, int offset) {
  int bits = (byte >> (offset * 2)) & 3;
  switch (bits) {
    case 0: return 2.0;
    case 1: return NAN;
    case 2: return 1.0;
    default: return 0.0;
  }
}

/* plink.rs:182-194 (raw row) and :237-247 (sample-subset gather). */
void orc_read_marker(const uint8_t* bed, int64_t bytes_per_marker, int64_t n_fam, int64_t marker,
                     const int64_t* sample_idx, int64_t n, double* dosages_out) {
  const uint8_t* row = bed + 3 + marker * bytes_per_marker;
  for (int64_t k = 0; k < n; ++k) {
    int64_t s = sample_idx ? sample_idx[k] : k;
    (void)n_fam;
    dosages_out[k] = orc_decode_genotype(row[s / 4], (int)(s % 4));
  }
}

/* saige-geno/src/traits.rs:42-54. */
void orc_compute_af(const double* dosages, int64_t n, double* af, double* mac, int64_t* n_valid) {
  double sum = 0.0;
  int64_t cnt = 0;
  for (int64_t i = 0; i < n; ++i) {
    double d = dosages[i];
    if (!isnan(d)) {
      sum += d;
      cnt += 1;
    }
  }
  *af = cnt > 0 ? sum / (2.0 * (double)cnt) : 0.0;
  double other = 2.0 * (double)cnt - sum;
  *mac = sum < other ? sum : other;
  *n_valid = cnt;
}

/* The read_marker + compute_af loop of fit_null.rs:209-211, with the bed
 * size checks of plink.rs:80-98.  Returns 0, or -1 on a malformed bed. */
int orc_marker_stats(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                     const int64_t* sample_idx, int64_t n, double* af, double* mac,
                     int64_t* n_valid) {
  if (bed_len < 3) return -1;
  if (bed[0] != 0x6C || bed[1] != 0x1B) return -1;
  if (bed[2] != 0x01) return -1;
  int64_t bpm = (n_fam + 3) / 4;
  if ((int64_t)bed_len < 3 + bpm * m_tot) return -1;
  for (int64_t k = 0; k < n; ++k)
    if (sample_idx && (sample_idx[k] < 0 || sample_idx[k] >= n_fam)) return -1;
#pragma omp parallel
  {
    double* dos = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(static)
    for (int64_t m = 0; m < m_tot; ++m) {
      orc_read_marker(bed, bpm, n_fam, m, sample_idx, n, dos);
      orc_compute_af(dos, n, &af[m], &mac[m], &n_valid[m]);
    }
    free(dos);
  }
  return 0;
}

/* ===================================================================== */
/* ChaCha (Bernstein's published specification) + rand 0.8.5 mappings    */
/* ===================================================================== */

static inline uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }

#define QR(a, b, c, d)            \
  do {                            \
    a += b; d ^= a; d = rotl32(d, 16); \
    c += d; b ^= c; b = rotl32(b, 12); \
    a += b; d ^= a; d = rotl32(d, 8);  \
    c += d; b ^= c; b = rotl32(b, 7);  \
  } while (0)

/* One 64-byte block: constants "expand 32-byte k", 8 key words, a 64-bit
 * block counter in words 12-13 and a 64-bit stream id in words 14-15 (the
 * layout rand_chacha uses).  rounds = 8 for ChaCha8, 20 for ChaCha20. */
void orc_chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds,
                      uint32_t out[16]) {
  uint32_t s[16];
  s[0] = 0x61707865u; s[1] = 0x3320646eu; s[2] = 0x79622d32u; s[3] = 0x6b206574u;
  for (int i = 0; i < 8; ++i) s[4 + i] = key[i];
  s[12] = (uint32_t)counter; s[13] = (uint32_t)(counter >> 32);
  s[14] = (uint32_t)stream;  s[15] = (uint32_t)(stream >> 32);
  uint32_t x[16];
  memcpy(x, s, sizeof x);
  for (int r = 0; r < rounds; r += 2) {
    QR(x[0], x[4], x[8], x[12]);
    QR(x[1], x[5], x[9], x[13]);
    QR(x[2], x[6], x[10], x[14]);
    QR(x[3], x[7], x[11], x[15]);
    QR(x[0], x[5], x[10], x[15]);
    QR(x[1], x[6], x[11], x[12]);
    QR(x[2], x[7], x[8], x[13]);
    QR(x[3], x[4], x[9], x[14]);
  }
  for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

void orc_chacha_from_seed(orc_chacha_rng* r, const uint8_t seed[32], int rounds) {
  for (int i = 0; i < 8; ++i)
    r->key[i] = (uint32_t)seed[4 * i] | ((uint32_t)seed[4 * i + 1] << 8) |
                ((uint32_t)seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
  r->counter = 0;
  r->stream = 0;
  r->idx = 64;
  r->rounds = rounds;
}

/* rand_core 0.6.4 SeedableRng::seed_from_u64: the 32-byte seed is filled
 * with successive PCG32 (XSH-RR) outputs, little-endian. */
void orc_chacha_seed_from_u64(orc_chacha_rng* r, uint64_t state, int rounds) {
  const uint64_t MUL = 6364136223846793005ull;
  const uint64_t INC = 11634580027462260723ull;
  uint8_t seed[32];
  for (int c = 0; c < 8; ++c) {
    state = state * MUL + INC;
    uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
    uint32_t rot = (uint32_t)(state >> 59);
    uint32_t x = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
    seed[4 * c] = (uint8_t)x; seed[4 * c + 1] = (uint8_t)(x >> 8);
    seed[4 * c + 2] = (uint8_t)(x >> 16); seed[4 * c + 3] = (uint8_t)(x >> 24);
  }
  orc_chacha_from_seed(r, seed, rounds);
}

static void orc_refill(orc_chacha_rng* r) {
  for (int b = 0; b < 4; ++b) orc_chacha_block(r->key, r->counter + b, r->stream, r->rounds, r->buf + 16 * b);
  r->counter += 4;
  r->idx = 0;
}

/* rand_core BlockRng: a contiguous stream of u32 words. */
uint32_t orc_rng_next_u32(orc_chacha_rng* r) {
  if (r->idx >= 64) orc_refill(r);
  return r->buf[r->idx++];
}

/* BlockRng::next_u64: two consecutive words, low word first (also across a
 * buffer refill). */
uint64_t orc_rng_next_u64(orc_chacha_rng* r) {
  uint64_t lo = orc_rng_next_u32(r);
  uint64_t hi = orc_rng_next_u32(r);
  return (hi << 32) | lo;
}

/* rand 0.8.5 Standard for bool: the sign bit of one u32. */
int orc_rng_gen_bool(orc_chacha_rng* r) { return (int32_t)orc_rng_next_u32(r) < 0; }

/* rand 0.8.5 UniformInt<u64/usize>::sample_single(low, high): widening
 * multiply with the "conservative zone" rejection test. */
uint64_t orc_rng_gen_range_u64(orc_chacha_rng* r, uint64_t low, uint64_t high) {
  uint64_t range = high - 1 - low + 1;
  if (range == 0) return orc_rng_next_u64(r);
  int lz = __builtin_clzll(range);
  uint64_t zone = (range << lz) - 1;
  for (;;) {
    uint64_t v = orc_rng_next_u64(r);
    unsigned __int128 prod = (unsigned __int128)v * (unsigned __int128)range;
    uint64_t hi = (uint64_t)(prod >> 64);
    uint64_t lo = (uint64_t)prod;
    if (lo <= zone) return low + hi;
  }
}

/* ai_reml.rs:121-130: n_vec Rademacher vectors from one ChaCha8 stream,
 * vector-major.  out is n_vec x n. */
void orc_rademacher_probes(uint64_t seed, int n_vec, int64_t n, double* out) {
  orc_chacha_rng r;
  orc_chacha_seed_from_u64(&r, seed, 8);
  for (int k = 0; k < n_vec; ++k)
    for (int64_t i = 0; i < n; ++i) out[(int64_t)k * n + i] = orc_rng_gen_bool(&r) ? 1.0 : -1.0;
}

/* ===================================================================== */
/* QC + VR/GRM split (saige-cli/src/commands/fit_null.rs:209-259)          */
/* ===================================================================== */

static int cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* Returns 0, or -1 when no marker passes QC (the reference panics in
 * gen_range(0..0)).  grm_idx / vr_idx receive original marker indices. */
int orc_select_markers(const double* af, const double* mac, const int64_t* n_valid, int64_t m_tot,
                       int64_t n, double min_maf, double max_missing, uint64_t seed,
                       int64_t* grm_idx, int64_t* m_grm, int64_t* vr_idx, int64_t* m_vr,
                       int64_t* n_pass_out) {
  int64_t* pass = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m_tot > 0 ? m_tot : 1));
  int64_t n_pass = 0;
  for (int64_t m = 0; m < m_tot; ++m) {
    double missing_rate = 1.0 - ((double)n_valid[m] / (double)n);
    if (af[m] >= min_maf && af[m] <= 1.0 - min_maf && missing_rate <= max_missing)
      pass[n_pass++] = m;
  }
  *n_pass_out = n_pass;
  if (n_pass == 0) {
    free(pass);
    *m_grm = 0;
    *m_vr = 0;
    return -1;
  }
  orc_chacha_rng r;
  orc_chacha_seed_from_u64(&r, seed, 8);
  uint64_t cand[1000];
  for (int k = 0; k < 1000; ++k) cand[k] = orc_rng_gen_range_u64(&r, 0, (uint64_t)n_pass);
  qsort(cand, 1000, sizeof(uint64_t), cmp_u64);
  unsigned char* is_vr = (unsigned char*)calloc((size_t)n_pass, 1);
  uint64_t prev = UINT64_MAX;
  for (int k = 0; k < 1000; ++k) {
    if (cand[k] == prev) continue;
    prev = cand[k];
    if (mac[pass[cand[k]]] >= 20.0) is_vr[cand[k]] = 1;
  }
  int64_t g = 0, v = 0;
  for (int64_t i = 0; i < n_pass; ++i) {
    if (is_vr[i]) vr_idx[v++] = pass[i];
    else grm_idx[g++] = pass[i];
  }
  *m_grm = g;
  *m_vr = v;
  free(is_vr);
  free(pass);
  return 0;
}

/* ===================================================================== */
/* On-the-fly GRM (saige-core/src/glmm/pcg.rs:91-180)                     */
/* ===================================================================== */

/* pcg.rs:101-122: z = (g - 2p)/sqrt(2p(1-p)) in f64, missing -> mean -> 0,
 * a column of zeros when the denominator is <= 1e-10.  mode 1 rounds to
 * f32 as the reference stores it.  z_out is m x n (marker-major). */
void orc_grm_standardize(const double* dosages, const double* af, int64_t n, int64_t m, int mode,
                         double* z_out) {
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < m; ++j) {
    double denom = sqrt(2.0 * af[j] * (1.0 - af[j]));
    double* zj = z_out + j * n;
    if (denom > 1e-10) {
      double mean = 2.0 * af[j];
      for (int64_t i = 0; i < n; ++i) {
        double g = dosages[j * n + i];
        if (isnan(g)) g = mean;
        double z = (g - mean) / denom;
        zj[i] = mode == 1 ? (double)(float)z : z;
      }
    } else {
      for (int64_t i = 0; i < n; ++i) zj[i] = 0.0;
    }
  }
}

/* pcg.rs:128-180.  mode 1 = the f32 arithmetic and the single-thread
 * sequential order (one rayon chunk: fold over markers, then x(1/M) in f32). */
void orc_grm_matvec(const double* z, int64_t n, int64_t m, const double* v, double* out, int mode) {
  if (m == 0) {
    for (int64_t i = 0; i < n; ++i) out[i] = 0.0;
    return;
  }
  if (mode == 1) {
    float* v32 = (float*)malloc(sizeof(float) * (size_t)n);
    float* acc = (float*)calloc((size_t)n, sizeof(float));
    float* z32 = (float*)malloc(sizeof(float) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) v32[i] = (float)v[i];
    for (int64_t j = 0; j < m; ++j) {
      for (int64_t i = 0; i < n; ++i) z32[i] = (float)z[j * n + i];
      float dot = 0.0f;
      for (int64_t i = 0; i < n; ++i) dot += z32[i] * v32[i];
      for (int64_t i = 0; i < n; ++i) acc[i] += z32[i] * dot;
    }
    float scale = 1.0f / (float)m;
    for (int64_t i = 0; i < n; ++i) out[i] = (double)(acc[i] * scale);
    free(v32); free(acc); free(z32);
    return;
  }
  double* dots = (double*)malloc(sizeof(double) * (size_t)m);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < m; ++j) {
    const double* zj = z + j * n;
    double d = 0.0;
    for (int64_t i = 0; i < n; ++i) d += zj[i] * v[i];
    dots[j] = d;
  }
  double scale = 1.0 / (double)m;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double a = 0.0;
    for (int64_t j = 0; j < m; ++j) a += z[j * n + i] * dots[j];
    out[i] = a * scale;
  }
  free(dots);
}

/* grm/dense.rs:115-186 semantics: K = Z'Z/M, n x n row-major, FP64. */
void orc_grm_explicit(const double* z, int64_t n, int64_t m, double* k_out) {
  double scale = m > 0 ? 1.0 / (double)m : 0.0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t a = 0; a < n; ++a) {
    for (int64_t b = a; b < n; ++b) {
      double s = 0.0;
      for (int64_t j = 0; j < m; ++j) s += z[j * n + a] * z[j * n + b];
      k_out[a * n + b] = s * scale;
      k_out[b * n + a] = s * scale;
    }
  }
}

int orc_grm_matvec_f32_packed(const uint8_t* bed_body, int64_t bpm, int64_t n,
                              const int64_t* rows, int64_t m, const double* af, const double* v,
                              double* out, int threads) {
  int nt = 1;
#ifdef _OPENMP
  nt = threads > 0 ? threads : omp_get_max_threads();
#endif
  float* v32 = (float*)malloc(sizeof(float) * (size_t)n);
  float* accs = (float*)calloc((size_t)n * (size_t)nt, sizeof(float));
  for (int64_t i = 0; i < n; ++i) v32[i] = (float)v[i];
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    float* acc = accs + (size_t)tid * (size_t)n;
#pragma omp for schedule(static)
    for (int64_t j = 0; j < m; ++j) {
      float lut[4] = {0.f, 0.f, 0.f, 0.f};
      const double p = af[j];
      const double denom = sqrt(2.0 * p * (1.0 - p));
      if (denom > 1e-10) {
        const double mean = 2.0 * p;
        lut[0] = (float)((2.0 - mean) / denom);
        lut[1] = 0.0f; /* missing -> mean -> 0 */
        lut[2] = (float)((1.0 - mean) / denom);
        lut[3] = (float)((0.0 - mean) / denom);
      }
      const uint8_t* row = bed_body + rows[j] * bpm;
      float dot = 0.0f;
      for (int64_t i = 0; i < n; ++i) dot += lut[(row[i >> 2] >> ((i & 3) * 2)) & 3] * v32[i];
      for (int64_t i = 0; i < n; ++i) acc[i] += lut[(row[i >> 2] >> ((i & 3) * 2)) & 3] * dot;
    }
  }
  const float scale = 1.0f / (float)m;
  for (int64_t i = 0; i < n; ++i) {
    float s = 0.0f;
    for (int t = 0; t < nt; ++t) s += accs[(size_t)t * (size_t)n + i];
    out[i] = (double)(s * scale);
  }
  free(v32);
  free(accs);
  return nt;
}

int orc_grm_matmul_f64_packed(const uint8_t* bed_body, int64_t bpm, int64_t n,
                              const int64_t* rows, int64_t m, const double* af, const double* v,
                              int nrhs, double* out) {
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  const int R = nrhs;
  double* lut = (double*)malloc(sizeof(double) * 4 * (size_t)(m > 0 ? m : 1));
  double* u = (double*)calloc((size_t)(m > 0 ? m : 1) * (size_t)R, sizeof(double));
  double* accs = (double*)calloc((size_t)n * (size_t)R * (size_t)nt, sizeof(double));
  for (int64_t j = 0; j < m; ++j) {
    const double p = af[j], denom = sqrt(2.0 * p * (1.0 - p));
    double* l = lut + 4 * j;
    l[0] = l[1] = l[2] = l[3] = 0.0;
    if (denom > 1e-10) {
      l[0] = (2.0 - 2.0 * p) / denom;
      l[2] = (1.0 - 2.0 * p) / denom;
      l[3] = (0.0 - 2.0 * p) / denom;
    }
  }
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    double* acc = accs + (size_t)tid * (size_t)n * (size_t)R;
    double d[64];
#pragma omp for schedule(dynamic, 16)
    for (int64_t j = 0; j < m; ++j) {
      const uint8_t* row = bed_body + rows[j] * bpm;
      const double* l = lut + 4 * j;
      for (int c = 0; c < R; ++c) d[c] = 0.0;
      for (int64_t i = 0; i < n; ++i) {
        const double z = l[(row[i >> 2] >> ((i & 3) * 2)) & 3];
        if (z != 0.0)
          for (int c = 0; c < R; ++c) d[c] += z * v[(int64_t)c * n + i];
      }
      for (int c = 0; c < R; ++c) u[j * R + c] = d[c];
      for (int64_t i = 0; i < n; ++i) {
        const double z = l[(row[i >> 2] >> ((i & 3) * 2)) & 3];
        if (z != 0.0)
          for (int c = 0; c < R; ++c) acc[(int64_t)c * n + i] += z * d[c];
      }
    }
  }
  const double scale = m > 0 ? 1.0 / (double)m : 0.0;
  for (int64_t k = 0; k < n * R; ++k) {
    double s = 0.0;
    for (int t = 0; t < nt; ++t) s += accs[(size_t)t * (size_t)n * (size_t)R + (size_t)k];
    out[k] = s * scale;
  }
  free(lut);
  free(u);
  free(accs);
  return nt;
}

/* ===================================================================== */
/* Dense linear algebra (saige-linalg/src/decomposition.rs)               */
/* ===================================================================== */

/* decomposition.rs:35-61; a and l are p x p row-major.  -1 = not PD. */
int orc_cholesky(const double* a, int p, double* l) {
  for (int i = 0; i < p * p; ++i) l[i] = 0.0;
  for (int j = 0; j < p; ++j) {
    double sum = 0.0;
    for (int k = 0; k < j; ++k) sum += l[j * p + k] * l[j * p + k];
    double diag = a[j * p + j] - sum;
    if (diag <= 0.0) return -1;
    l[j * p + j] = sqrt(diag);
    for (int i = j + 1; i < p; ++i) {
      double s = 0.0;
      for (int k = 0; k < j; ++k) s += l[i * p + k] * l[j * p + k];
      l[i * p + j] = (a[i * p + j] - s) / l[j * p + j];
    }
  }
  return 0;
}

/* decomposition.rs:64-89. */
void orc_chol_solve(const double* l, int p, const double* b, double* x) {
  double y[64];
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

typedef void (*orc_op_fn)(void* ctx, const double* v, double* out);

/* decomposition.rs:212-298, verbatim control flow: x0 (or 0), r = b - A x,
 * tol_abs = tol * max(||b||, 1), test ||r|| before each product, give up
 * when |p'Ap| < 1e-30.  Returns 1 when converged. */
static int orc_pcg_core(orc_op_fn op, void* op_ctx, orc_op_fn pre, void* pre_ctx, int64_t n,
                        const double* b, const double* x0, double tol, int max_iter, double* x,
                        int* iters, double* resid) {
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  double* z = (double*)malloc(sizeof(double) * (size_t)n);
  double* p = (double*)malloc(sizeof(double) * (size_t)n);
  double* ap = (double*)malloc(sizeof(double) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) x[i] = x0 ? x0[i] : 0.0;
  op(op_ctx, x, ap);
  for (int64_t i = 0; i < n; ++i) r[i] = b[i] - ap[i];
  pre(pre_ctx, r, z);
  for (int64_t i = 0; i < n; ++i) p[i] = z[i];
  double rz = 0.0;
  for (int64_t i = 0; i < n; ++i) rz += r[i] * z[i];
  double bn = 0.0;
  for (int64_t i = 0; i < n; ++i) bn += b[i] * b[i];
  bn = sqrt(bn);
  double tol_abs = tol * (bn > 1.0 ? bn : 1.0);
  int conv = 0;
  int it;
  double rn = 0.0;
  for (it = 0; it < max_iter; ++it) {
    rn = 0.0;
    for (int64_t i = 0; i < n; ++i) rn += r[i] * r[i];
    rn = sqrt(rn);
    if (rn < tol_abs) { conv = 1; break; }
    op(op_ctx, p, ap);
    double pap = 0.0;
    for (int64_t i = 0; i < n; ++i) pap += p[i] * ap[i];
    if (fabs(pap) < 1e-30) { conv = 0; goto done; }
    double alpha = rz / pap;
    for (int64_t i = 0; i < n; ++i) x[i] += alpha * p[i];
    for (int64_t i = 0; i < n; ++i) r[i] -= alpha * ap[i];
    pre(pre_ctx, r, z);
    double rz_new = 0.0;
    for (int64_t i = 0; i < n; ++i) rz_new += r[i] * z[i];
    double beta = rz_new / rz;
    rz = rz_new;
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  if (!conv) {
    rn = 0.0;
    for (int64_t i = 0; i < n; ++i) rn += r[i] * r[i];
    rn = sqrt(rn);
    conv = rn < tol_abs;
    it = max_iter;
  }
done:
  *iters = it;
  *resid = rn;
  free(r); free(z); free(p); free(ap);
  return conv;
}

typedef struct { const double* a; int n; } dense_ctx;
static void dense_op(void* c, const double* v, double* out) {
  dense_ctx* d = (dense_ctx*)c;
  for (int i = 0; i < d->n; ++i) out[i] = 0.0;
  /* DenseMatrix::mat_vec (dense.rs:102-113): column sweep */
  for (int j = 0; j < d->n; ++j)
    for (int i = 0; i < d->n; ++i) out[i] += d->a[i * d->n + j] * v[j];
}
static void dense_diag_pre(void* c, const double* v, double* out) {
  dense_ctx* d = (dense_ctx*)c;
  for (int i = 0; i < d->n; ++i) {
    double di = d->a[i * d->n + i];
    out[i] = fabs(di) > 1e-30 ? v[i] / di : v[i];
  }
}

/* decomposition.rs:301-315 (solve_dense: Jacobi on diag(A)).  Returns 1 when
 * converged; a is n x n row-major. */
int orc_pcg_dense(const double* a, int n, const double* b, double tol, int max_iter, double* x,
                  int* iters, double* resid) {
  dense_ctx c = {a, n};
  return orc_pcg_core(dense_op, &c, dense_diag_pre, &c, n, b, NULL, tol, max_iter, x, iters, resid);
}

/* ===================================================================== */
/* Link and family (saige-core/src/glmm/link.rs:29-100, family.rs:23-90)  */
/* ===================================================================== */

double orc_link(int t, double mu) {
  if (t == ORC_BINARY) return log(mu / (1.0 - mu));
  if (t == ORC_QUANTITATIVE) return mu;
  return log(-log(1.0 - mu));
}
double orc_inv_link(int t, double eta) {
  if (t == ORC_BINARY) return 1.0 / (1.0 + exp(-eta));
  if (t == ORC_QUANTITATIVE) return eta;
  return 1.0 - exp(-exp(eta));
}
/* family.rs:82-90: clamp to [1e-10, 1-1e-10] for binary/survival. */
double orc_update_mu(int t, double eta) {
  double mu = orc_inv_link(t, eta);
  if (t == ORC_QUANTITATIVE) return mu;
  if (mu < 1e-10) mu = 1e-10;
  if (mu > 1.0 - 1e-10) mu = 1.0 - 1e-10;
  return mu;
}
/* family.rs:55-66 with link.rs variance(). */
double orc_working_weight(int t, double mu) {
  double v = t == ORC_QUANTITATIVE ? 1.0 : mu * (1.0 - mu);
  return v > 1e-30 ? v : 1e-30;
}
/* family.rs:23-40. */
double orc_initialize_mu(int t, double y) {
  if (t == ORC_BINARY) return (y + 0.5) / 2.0;
  if (t == ORC_QUANTITATIVE) return y;
  double m = (y + 0.5) / 2.0;
  if (m < 0.01) m = 0.01;
  if (m > 0.99) m = 0.99;
  return m;
}

/* ===================================================================== */
/* GLM IRLS (ai_reml.rs:431-482)                                          */
/* ===================================================================== */

/* x is n x p column-major (DenseMatrix::from_col_major). */
int orc_fit_glm_irls(const double* y, const double* x, int64_t n, int p, int t, int max_iter,
                     double* alpha) {
  double* mu = (double*)malloc(sizeof(double) * (size_t)n);
  double* eta = (double*)malloc(sizeof(double) * (size_t)n);
  double* w = (double*)malloc(sizeof(double) * (size_t)n);
  double* zz = (double*)malloc(sizeof(double) * (size_t)n);
  double xtwx[64 * 64], l[64 * 64], xtwz[64], anew[64];
  int rc = 0;
  for (int64_t i = 0; i < n; ++i) {
    mu[i] = orc_initialize_mu(t, y[i]);
    eta[i] = orc_link(t, mu[i]);
  }
  for (int j = 0; j < p; ++j) alpha[j] = 0.0;
  for (int it = 0; it < max_iter; ++it) {
    for (int64_t i = 0; i < n; ++i) {
      w[i] = orc_working_weight(t, mu[i]);
      double wm = w[i] > 1e-30 ? w[i] : 1e-30;
      zz[i] = eta[i] + (y[i] - mu[i]) / wm;
    }
    /* dense.rs:227-263 */
    for (int j = 0; j < p; ++j)
      for (int k = j; k < p; ++k) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += x[j * n + i] * w[i] * x[k * n + i];
        xtwx[j * p + k] = s;
        xtwx[k * p + j] = s;
      }
    for (int j = 0; j < p; ++j) {
      double s = 0.0;
      for (int64_t i = 0; i < n; ++i) s += x[j * n + i] * w[i] * zz[i];
      xtwz[j] = s;
    }
    if (orc_cholesky(xtwx, p, l) != 0) {
      for (int i = 0; i < p; ++i) xtwx[i * p + i] += 1e-6;
      if (orc_cholesky(xtwx, p, l) != 0) { rc = -1; break; }
    }
    orc_chol_solve(l, p, xtwz, anew);
    /* DenseMatrix::mat_vec: column sweep */
    for (int64_t i = 0; i < n; ++i) eta[i] = 0.0;
    for (int j = 0; j < p; ++j)
      for (int64_t i = 0; i < n; ++i) eta[i] += x[j * n + i] * anew[j];
    for (int64_t i = 0; i < n; ++i) mu[i] = orc_update_mu(t, eta[i]);
    double change = 0.0;
    for (int j = 0; j < p; ++j) change += fabs(anew[j] - alpha[j]);
    for (int j = 0; j < p; ++j) alpha[j] = anew[j];
    if (change < 1e-8) break;
  }
  free(mu); free(eta); free(w); free(zz);
  return rc;
}

/* ===================================================================== */
/* AI-REML (ai_reml.rs:86-427)                                            */
/* ===================================================================== */

typedef struct {
  int kind;
  const double* grm;
  int64_t n, m;
  int kmode;
  int64_t n_kv;
  float* z32;  /* kmode 2: Z as f32, built once per fit (OnTheFlyGrm::new, pcg.rs:101-122) */
} grm_ctx;

/* kmode 2 of ORC_K_OTF: the saige-rs product as it runs, on all host threads —
 * f32 Z (marker-major), per marker an f32 dot then an f32 axpy into the thread's
 * accumulator, chunks of >= 64 markers per task (the rayon fold of pcg.rs:149-169),
 * the per-thread accumulators summed in f32 (the reduce, :170-176), then x(1/M). */
static void grm_matvec_f32_parallel(const float* z32, int64_t n, int64_t m, const double* v,
                                    double* out) {
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  float* v32 = (float*)malloc(sizeof(float) * (size_t)n);
  float* accs = (float*)calloc((size_t)n * (size_t)nt, sizeof(float));
  for (int64_t i = 0; i < n; ++i) v32[i] = (float)v[i];
#pragma omp parallel num_threads(nt)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    float* acc = accs + (size_t)tid * (size_t)n;
#pragma omp for schedule(dynamic, 64)
    for (int64_t j = 0; j < m; ++j) {
      const float* zj = z32 + j * n;
      float dot = 0.0f;
      for (int64_t i = 0; i < n; ++i) dot += zj[i] * v32[i];
      for (int64_t i = 0; i < n; ++i) acc[i] += zj[i] * dot;
    }
  }
  const float scale = 1.0f / (float)m;
  for (int64_t i = 0; i < n; ++i) {
    float s = 0.0f;
    for (int t = 0; t < nt; ++t) s += accs[(size_t)t * (size_t)n + i];
    out[i] = (double)(s * scale);
  }
  free(v32);
  free(accs);
}

static void grm_ctx_init(grm_ctx* g, int kind, const double* grm, int64_t n, int64_t m,
                         int kmode) {
  g->kind = kind;
  g->grm = grm;
  g->n = n;
  g->m = m;
  g->kmode = kmode;
  g->n_kv = 0;
  g->z32 = NULL;
  if (kind == ORC_K_OTF && kmode == 2 && m > 0) {
    g->z32 = (float*)malloc(sizeof(float) * (size_t)n * (size_t)m);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n * m; ++k) g->z32[k] = (float)grm[k];
  }
}

static void grm_apply(grm_ctx* g, const double* v, double* out) {
  g->n_kv += 1;
  if (g->kind == ORC_K_IDENTITY) {
    for (int64_t i = 0; i < g->n; ++i) out[i] = v[i];
  } else if (g->kind == ORC_K_OTF && g->z32) {
    grm_matvec_f32_parallel(g->z32, g->n, g->m, v, out);
  } else if (g->kind == ORC_K_OTF) {
    orc_grm_matvec(g->grm, g->n, g->m, v, out, g->kmode);
  } else {
    int64_t n = g->n;
#pragma omp parallel for schedule(static)
    for (int64_t a = 0; a < n; ++a) {
      double s = 0.0;
      const double* row = g->grm + a * n;
      for (int64_t b = 0; b < n; ++b) s += row[b] * v[b];
      out[a] = s;
    }
  }
}

typedef struct {
  grm_ctx* g;
  const double* w;
  double tau0, tau1;
  double* tmp;
} sigma_ctx;

/* ai_reml.rs:142-149 */
static void sigma_op(void* c, const double* v, double* out) {
  sigma_ctx* s = (sigma_ctx*)c;
  grm_apply(s->g, v, s->tmp);
  for (int64_t i = 0; i < s->g->n; ++i) {
    double wi = s->w[i] > 1e-30 ? s->w[i] : 1e-30;
    out[i] = s->tau0 * v[i] / wi + s->tau1 * s->tmp[i];
  }
}
/* ai_reml.rs:152-164 */
static void sigma_pre(void* c, const double* v, double* out) {
  sigma_ctx* s = (sigma_ctx*)c;
  for (int64_t i = 0; i < s->g->n; ++i) {
    double wi = s->w[i] > 1e-30 ? s->w[i] : 1e-30;
    double diag = s->tau0 / wi + s->tau1;
    out[i] = fabs(diag) > 1e-30 ? v[i] / diag : v[i];
  }
}

int orc_pcg_sigma(const double* y_unused, int kind, const double* grm, int64_t n, int64_t m,
                  int kmode, const double* w, const double tau[2], const double* b,
                  const double* x0, double tol, int max_iter, double* x, int* iters,
                  double* resid, int* converged) {
  (void)y_unused;
  grm_ctx g;
  grm_ctx_init(&g, kind, grm, n, m, kmode);
  double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
  sigma_ctx s = {&g, w, tau[0], tau[1], tmp};
  *converged = orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, b, x0, tol, max_iter, x, iters, resid);
  free(tmp);
  free(g.z32);
  return 0;
}

static double dotv(const double* a, const double* b, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* P-projection of a Sigma^-1 solve (ai_reml.rs:242-251):
 * pu = sinv_u - SinvX C^-1 (SinvX' u). */
static void p_project(double* pu, const double* u, const double* sinvx, const double* l, int p,
                      int64_t n) {
  double t[64], corr[64];
  for (int j = 0; j < p; ++j) t[j] = dotv(sinvx + (int64_t)j * n, u, n);
  orc_chol_solve(l, p, t, corr);
  for (int j = 0; j < p; ++j)
    for (int64_t i = 0; i < n; ++i) pu[i] -= sinvx[(int64_t)j * n + i] * corr[j];
}

int orc_fit_ai_reml(const double* y, const double* x, int64_t n, int p, int t, int kind,
                    const double* grm, int64_t m, int kmode, const orc_ai_reml_config* cfg,
                    orc_ai_reml_summary* out, double* tau_trace, double* alpha_out,
                    double* mu_out, double* eta_out, double* w_out) {
  if (p > 64) return -2;
  int fix_tau_e = (t == ORC_BINARY || t == ORC_SURVIVAL);
  double tau[2] = {1.0, 0.0};
  double alpha[64];
  if (orc_fit_glm_irls(y, x, n, p, t, 25, alpha) != 0) return -1;

  size_t nb = sizeof(double) * (size_t)n;
  double* eta = (double*)malloc(nb);
  double* mu = (double*)malloc(nb);
  double* w = (double*)malloc(nb);
  double* ytil = (double*)malloc(nb);
  double* sinvy = (double*)malloc(nb);
  double* sinvx = (double*)malloc(nb * (size_t)p);
  double* xcol = (double*)malloc(nb);
  double* py = (double*)malloc(nb);
  double* kpy = (double*)malloc(nb);
  double* su = (double*)malloc(nb);
  double* ku = (double*)malloc(nb);
  double* pk = (double*)malloc(nb);
  double* invw_py = (double*)malloc(nb);
  double* tmp = (double*)malloc(nb);
  int nrv = cfg->n_random_vectors;
  double* probes = (double*)malloc(nb * (size_t)(nrv > 0 ? nrv : 1));
  orc_rademacher_probes(cfg->seed, nrv, n, probes);

  for (int64_t i = 0; i < n; ++i) {
    double e = 0.0;
    for (int j = 0; j < p; ++j) e += x[(int64_t)j * n + i] * alpha[j];
    eta[i] = e;
    mu[i] = orc_update_mu(t, e);
  }

  grm_ctx g;
  grm_ctx_init(&g, kind, grm, n, m, kmode);
  int64_t pcg_total = 0;
  int converged = 0, n_iter = 0;
  double l[64 * 64], c[64 * 64];

  for (int iter = 0; iter < cfg->max_iter; ++iter) {
    n_iter = iter + 1;
    for (int64_t i = 0; i < n; ++i) w[i] = orc_working_weight(t, mu[i]);
    sigma_ctx s = {&g, w, tau[0], tau[1], tmp};
    for (int64_t i = 0; i < n; ++i) {
      double wi = w[i] > 1e-30 ? w[i] : 1e-30;
      ytil[i] = eta[i] + (y[i] - mu[i]) / wi;
    }
    int it;
    double rs;
    orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, ytil, NULL, cfg->pcg_tol, cfg->pcg_max_iter,
                 sinvy, &it, &rs);
    pcg_total += it;
    for (int j = 0; j < p; ++j) {
      for (int64_t i = 0; i < n; ++i) xcol[i] = x[(int64_t)j * n + i];
      orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, xcol, NULL, cfg->pcg_tol, cfg->pcg_max_iter,
                   sinvx + (int64_t)j * n, &it, &rs);
      pcg_total += it;
    }
    /* ai_reml.rs:189-200: C[j,k] = X[:,k] . SinvX[:,j] */
    for (int j = 0; j < p; ++j)
      for (int k = j; k < p; ++k) {
        double d = dotv(x + (int64_t)k * n, sinvx + (int64_t)j * n, n);
        c[j * p + k] = d;
        c[k * p + j] = d;
      }
    double xsy[64];
    for (int j = 0; j < p; ++j) xsy[j] = dotv(x + (int64_t)j * n, sinvy, n);
    if (orc_cholesky(c, p, l) != 0) break;
    orc_chol_solve(l, p, xsy, alpha);
    for (int64_t i = 0; i < n; ++i) {
      double e = 0.0;
      for (int j = 0; j < p; ++j) e += x[(int64_t)j * n + i] * alpha[j];
      eta[i] = e;
      mu[i] = orc_update_mu(t, e);
    }
    /* ai_reml.rs:221-232 */
    for (int64_t i = 0; i < n; ++i) py[i] = sinvy[i];
    for (int j = 0; j < p; ++j)
      for (int64_t i = 0; i < n; ++i) py[i] -= sinvx[(int64_t)j * n + i] * alpha[j];
    grm_apply(&g, py, kpy);
    double ypapy = dotv(py, kpy, n);
    /* ai_reml.rs:237-258: Hutchinson trace of P K */
    double trace_sum = 0.0;
    for (int k = 0; k < nrv; ++k) {
      const double* u = probes + (int64_t)k * n;
      orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, u, NULL, cfg->pcg_tol, cfg->pcg_max_iter, su,
                   &it, &rs);
      pcg_total += it;
      p_project(su, u, sinvx, l, p, n);
      grm_apply(&g, u, ku);
      trace_sum += dotv(ku, su, n);
    }
    double trace_grm = trace_sum / (double)nrv;
    double score_g = ypapy - trace_grm;
    /* ai_reml.rs:263-273 */
    orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, kpy, NULL, cfg->pcg_tol, cfg->pcg_max_iter, pk,
                 &it, &rs);
    pcg_total += it;
    p_project(pk, kpy, sinvx, l, p, n);
    double ai_11 = dotv(kpy, pk, n);
    double score_e = 0.0, ai_00 = 0.0, ai_01 = 0.0;
    if (!fix_tau_e) {
      /* ai_reml.rs:281-317 */
      double tw = 0.0;
      for (int k = 0; k < nrv; ++k) {
        const double* u = probes + (int64_t)k * n;
        orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, u, NULL, cfg->pcg_tol, cfg->pcg_max_iter, su,
                     &it, &rs);
        pcg_total += it;
        p_project(su, u, sinvx, l, p, n);
        double d = 0.0;
        for (int64_t i = 0; i < n; ++i) {
          double wi = w[i] > 1e-30 ? w[i] : 1e-30;
          d += (u[i] / wi) * su[i];
        }
        tw += d;
      }
      double trace_w = tw / (double)nrv;
      for (int64_t i = 0; i < n; ++i) {
        double wi = w[i] > 1e-30 ? w[i] : 1e-30;
        invw_py[i] = py[i] / wi;
      }
      double ypa0py = dotv(py, invw_py, n);
      score_e = ypa0py - trace_w;
      orc_pcg_core(sigma_op, &s, sigma_pre, &s, n, invw_py, NULL, cfg->pcg_tol,
                   cfg->pcg_max_iter, su, &it, &rs);
      pcg_total += it;
      p_project(su, invw_py, sinvx, l, p, n);
      ai_00 = dotv(invw_py, su, n);
      ai_01 = dotv(invw_py, pk, n);
    }
    double tau_new[2], max_change;
    if (fix_tau_e) {
      if (fabs(ai_11) < 1e-30) break;
      double d1 = score_g / ai_11;
      double step = 1.0;
      double tg = tau[1] + step * d1;
      while (tg < 0.0 && step > 1e-10) {
        step *= 0.5;
        tg = tau[1] + step * d1;
      }
      if (tg < 1e-10) tg = 1e-10;
      max_change = fabs(tg - tau[1]) / (fabs(tg) + fabs(tau[1]) + cfg->tol);
      tau_new[0] = 1.0;
      tau_new[1] = tg;
    } else {
      double det = ai_00 * ai_11 - ai_01 * ai_01;
      if (fabs(det) < 1e-30) break;
      double d0 = (ai_11 * score_e - ai_01 * score_g) / det;
      double d1 = (-ai_01 * score_e + ai_00 * score_g) / det;
      double step = 1.0;
      double t0 = tau[0] + step * d0, t1 = tau[1] + step * d1;
      while ((t0 < 0.0 || t1 < 0.0) && step > 1e-10) {
        step *= 0.5;
        t0 = tau[0] + step * d0;
        t1 = tau[1] + step * d1;
      }
      tau_new[0] = t0 > 1e-10 ? t0 : 1e-10;
      tau_new[1] = t1 > 1e-10 ? t1 : 1e-10;
      double c0 = fabs(tau_new[0] - tau[0]) / (fabs(tau_new[0]) + fabs(tau[0]) + cfg->tol);
      double c1 = fabs(tau_new[1] - tau[1]) / (fabs(tau_new[1]) + fabs(tau[1]) + cfg->tol);
      max_change = c0 > c1 ? c0 : c1;
    }
    tau[0] = tau_new[0];
    tau[1] = tau_new[1];
    if (tau_trace) {
      tau_trace[2 * iter] = tau[0];
      tau_trace[2 * iter + 1] = tau[1];
    }
    if (max_change < cfg->tol) {
      converged = 1;
      break;
    }
  }
  for (int64_t i = 0; i < n; ++i) w[i] = orc_working_weight(t, mu[i]);
  double ll = 0.0;
  if (t == ORC_QUANTITATIVE) {
    double ss = 0.0;
    for (int64_t i = 0; i < n; ++i) ss += (y[i] - mu[i]) * (y[i] - mu[i]);
    ll = -0.5 * (double)n * log(2.0 * M_PI * tau[0]) - 0.5 * ss / tau[0];
  } else {
    for (int64_t i = 0; i < n; ++i) {
      double mi = mu[i];
      if (mi < 1e-15) mi = 1e-15;
      if (mi > 1.0 - 1e-15) mi = 1.0 - 1e-15;
      ll += y[i] * log(mi) + (1.0 - y[i]) * log(1.0 - mi);
    }
  }
  out->tau[0] = tau[0];
  out->tau[1] = tau[1];
  out->iterations = n_iter;
  out->converged = converged;
  out->log_likelihood = ll;
  out->n_kv = g.n_kv;
  out->pcg_iters = pcg_total;
  if (alpha_out) for (int j = 0; j < p; ++j) alpha_out[j] = alpha[j];
  if (mu_out) memcpy(mu_out, mu, nb);
  if (eta_out) memcpy(eta_out, eta, nb);
  if (w_out) memcpy(w_out, w, nb);
  free(eta); free(mu); free(w); free(ytil); free(sinvy); free(sinvx); free(xcol); free(py);
  free(kpy); free(su); free(ku); free(pk); free(invw_py); free(tmp); free(probes);
  free(g.z32);
  return 0;
}


/* ===================================================================== */
/* Variance ratio (saige-core/src/glmm/variance_ratio.rs:87-246,         */
/* saige-cli/src/commands/fit_null.rs:290-373)                            */
/* ===================================================================== */

/* rand 0.8.5 UniformInt<u32>::sample_single(low, high) -> sample_single_inclusive(low, high-1):
 * range = high - low, zone = (range << lz) - 1, v = next_u32, accept when the low half of
 * v * range is <= zone and return low + the high half. */
uint32_t orc_rng_gen_range_u32(orc_chacha_rng* r, uint32_t low, uint32_t high) {
  uint32_t range = high - low;
  uint32_t zone = (range << __builtin_clz(range)) - 1u;
  for (;;) {
    uint64_t prod = (uint64_t)orc_rng_next_u32(r) * (uint64_t)range;
    if ((uint32_t)prod <= zone) return low + (uint32_t)(prod >> 32);
  }
}

/* rand 0.8.5 SliceRandom::shuffle: for i = len-1 down to 1, swap(i, gen_index(i+1)) with
 * gen_index using the u32 range when the bound fits in 32 bits (variance_ratio.rs:116-120). */
void orc_shuffled_indices(uint64_t seed, int64_t len, int64_t* out) {
  orc_chacha_rng r;
  orc_chacha_seed_from_u64(&r, seed, 8);
  for (int64_t i = 0; i < len; ++i) out[i] = i;
  for (int64_t i = len - 1; i >= 1; --i) {
    uint64_t ub = (uint64_t)i + 1;
    int64_t j = ub <= 0xFFFFFFFFull ? (int64_t)orc_rng_gen_range_u32(&r, 0, (uint32_t)ub)
                                    : (int64_t)orc_rng_gen_range_u64(&r, 0, ub);
    int64_t t = out[i];
    out[i] = out[j];
    out[j] = t;
  }
}

/* variance_ratio.rs:260-272: (sd / mean) / n, infinity for n <= 1 or |mean| < 1e-30. */
static double vr_cal_cv(const double* v, int n) {
  if (n <= 1) return INFINITY;
  double m = 0.0;
  for (int i = 0; i < n; ++i) m += v[i];
  m /= (double)n;
  if (fabs(m) < 1e-30) return INFINITY;
  double var = 0.0;
  for (int i = 0; i < n; ++i) var += (v[i] - m) * (v[i] - m);
  var /= ((double)n - 1.0);
  return (sqrt(var) / m) / (double)n;
}

int orc_variance_ratio(const double* dosages, const double* mac, int64_t n_cand, const double* mu,
                       const double* w, const double tau[2], int t, const double* x, int64_t n,
                       int p, int kind, const double* grm, int64_t m, int kmode,
                       const orc_vr_config* cfg, orc_vr_summary* out, double* per_marker_vr,
                       int64_t* used_idx) {
  /* fit_null.rs:290-306: XVX = X'WX (dense.rs:227-245), its inverse (inverse_spd:
   * Cholesky, unit columns), and XVX_inv_XV filled as data[j*n + i]. */
  double xvx[64 * 64] = {0}, l[64 * 64], inv[64 * 64];
  for (int j = 0; j < p; ++j)
    for (int k = j; k < p; ++k) {
      double s = 0.0;
      for (int64_t i = 0; i < n; ++i) s += x[(int64_t)j * n + i] * w[i] * x[(int64_t)k * n + i];
      xvx[j * p + k] = s;
      xvx[k * p + j] = s;
    }
  if (orc_cholesky(xvx, p, l) != 0) return 2;
  for (int j = 0; j < p; ++j) {
    double e[64], col[64];
    for (int k = 0; k < p; ++k) e[k] = k == j ? 1.0 : 0.0;
    orc_chol_solve(l, p, e, col);
    for (int k = 0; k < p; ++k) inv[k * p + j] = col[k];  /* inv(k, j) */
  }
  double* data = (double*)malloc(sizeof(double) * (size_t)p * (size_t)n);
  for (int j = 0; j < p; ++j)
    for (int64_t i = 0; i < n; ++i) {
      double val = 0.0;
      for (int k = 0; k < p; ++k) val += inv[j * p + k] * x[(int64_t)k * n + i] * w[i];
      data[(int64_t)j * n + i] = val;
    }

  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n_cand > 0 ? n_cand : 1));
  orc_shuffled_indices(cfg->seed, n_cand, order);
  double* g0 = (double*)malloc(sizeof(double) * (size_t)n);
  double* gt = (double*)malloc(sizeof(double) * (size_t)n);
  double* sg = (double*)malloc(sizeof(double) * (size_t)n);
  int n_tested = 0, target = cfg->n_markers;
  int64_t n_kv = 0;
  for (int64_t oi = 0; oi < n_cand; ++oi) {
    const int64_t idx = order[oi];
    if (mac[idx] < cfg->min_mac) continue;
    const double* g_raw = dosages + idx * n;
    /* missing calls -> 2 * af of the called genotypes (see the header) */
    double s_nm = 0.0;
    int64_t n_nm = 0;
    for (int64_t i = 0; i < n; ++i)
      if (!isnan(g_raw[i])) { s_nm += g_raw[i]; ++n_nm; }
    const double fill = n_nm > 0 ? 2.0 * (s_nm / (2.0 * (double)n_nm)) : 0.0;
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      g0[i] = isnan(g_raw[i]) ? fill : g_raw[i];
      sum += g0[i];
    }
    const double af = sum / (2.0 * (double)n);
    if (af > 0.5)
      for (int64_t i = 0; i < n; ++i) g0[i] = 2.0 - g0[i];
    double ac = 0.0;
    for (int64_t i = 0; i < n; ++i) ac += g0[i];
    if (ac < 1.0) continue;
    /* X-adjust (variance_ratio.rs:144-151) */
    double tcoef[64];
    for (int r = 0; r < p; ++r) tcoef[r] = 0.0;
    if (cfg->xadjust == 0) {
      /* DenseMatrix::from_col_major(p, n, data).mat_vec(g0) (dense.rs:35-38, 102-113):
       * element (r, c) = data[c * p + r], accumulated column by column */
      for (int64_t c = 0; c < n; ++c) {
        const double vc = g0[c];
        for (int r = 0; r < p; ++r) tcoef[r] += data[c * p + r] * vc;
      }
    } else {
      for (int r = 0; r < p; ++r) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += data[(int64_t)r * n + i] * g0[i];
        tcoef[r] = s;
      }
    }
    /* x.mat_vec(t) column by column, then g_tilde = g0 - X t */
    for (int64_t i = 0; i < n; ++i) sg[i] = 0.0;
    for (int k = 0; k < p; ++k)
      for (int64_t i = 0; i < n; ++i) sg[i] += x[(int64_t)k * n + i] * tcoef[k];
    for (int64_t i = 0; i < n; ++i) gt[i] = g0[i] - sg[i];
    /* Sigma^-1 g_tilde: PcgSolver::new(1e-5, 500), zero start (fit_null.rs:317-342) */
    int iters = 0, conv = 0;
    double resid = 0.0;
    orc_pcg_sigma(NULL, kind, grm, n, m, kmode, w, tau, gt, NULL, 1e-5, 500, sg, &iters, &resid,
                  &conv);
    n_kv += iters;
    double var1 = 0.0;
    for (int64_t i = 0; i < n; ++i) var1 += gt[i] * sg[i];
    var1 /= ac;
    double var2 = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      /* variance_ratio.rs:162-180 */
      const double c = t == ORC_BINARY ? mu[i] * (1.0 - mu[i]) : (t == ORC_SURVIVAL ? mu[i] : 1.0);
      var2 += c * gt[i] * gt[i] / ac;
    }
    if (var2 < 1e-30) continue;
    per_marker_vr[n_tested] = var1 / var2;
    if (used_idx) used_idx[n_tested] = idx;
    ++n_tested;
    if (n_tested >= target) {
      if (vr_cal_cv(per_marker_vr, n_tested) <= cfg->ratio_cv_cutoff) break;
      target += 10;
    }
  }
  free(order); free(g0); free(gt); free(sg); free(data);
  out->n_kv = n_kv;
  out->n_markers_used = n_tested;
  out->n_categories = 0;
  if (n_tested == 0) return 1;
  double mean = 0.0;
  for (int i = 0; i < n_tested; ++i) mean += per_marker_vr[i];
  out->variance_ratio = mean / (double)n_tested;
  if (cfg->use_categorical) {
    /* variance_ratio.rs:276-298 with the default MAC bins */
    static const double lo[8] = {0.5, 1.5, 2.5, 3.5, 4.5, 5.5, 10.5, 20.5};
    static const double hi[8] = {1.5, 2.5, 3.5, 4.5, 5.5, 10.5, 20.5, INFINITY};
    for (int b = 0; b < 8; ++b) {
      double s = 0.0;
      int c = 0;
      for (int i = 0; i < n_tested; ++i) {
        const double mc = mac[used_idx ? used_idx[i] : 0];
        if (mc > lo[b] && mc <= hi[b]) { s += per_marker_vr[i]; ++c; }
      }
      if (c > 0) {
        out->cat_upper[out->n_categories] = hi[b];
        out->cat_vr[out->n_categories] = s / (double)c;
        ++out->n_categories;
      }
    }
  }
  return 0;
}

/* ===================================================================== */
/* Explicit GRM (saige-core/src/grm/dense.rs)                             */
/* ===================================================================== */

/* The accumulation of dense.rs:66-86 / :147-163 and the scaling of :89-102 /
 * :165-177, in the reference's loop order: row i keeps row_vals[j - i] for
 * j >= i and adds gi * z_j for every used marker in turn, so each K_ij (i <= j)
 * is one f64 sum over the markers in order (multiply, then add); the result is
 * multiplied by 1/n_used and mirrored. */
static void orc_grm_accumulate(const double* z, int64_t n, int64_t n_used, double* out) {
  const double scale = n_used > 0 ? 1.0 / (double)n_used : 0.0;
#pragma omp parallel
  {
    double* row_vals = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
#pragma omp for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; ++i) {
      const int64_t len = n - i;
      for (int64_t k = 0; k < len; ++k) row_vals[k] = 0.0;
      for (int64_t mk = 0; mk < n_used; ++mk) {
        const double* zk = z + mk * n;
        const double gi = zk[i];
        for (int64_t k = 0; k < len; ++k) row_vals[k] += gi * zk[i + k];
      }
      for (int64_t k = 0; k < len; ++k) {
        const double v = n_used > 0 ? row_vals[k] * scale : 0.0;
        out[i * n + i + k] = v;
        out[(i + k) * n + i] = v;
      }
    }
    free(row_vals);
  }
}

/* dense.rs:46-58 / :129-140: standardise one marker; returns 0 when skipped. */
static int orc_grm_std_marker(const double* d, int64_t n, double af, double* z) {
  const double var = 2.0 * af * (1.0 - af);
  if (var < 1e-10) return 0;
  const double sd = sqrt(var);
  const double mean = 2.0 * af;
  for (int64_t i = 0; i < n; ++i) {
    const double di = isnan(d[i]) ? mean : d[i];
    z[i] = (di - mean) / sd;
  }
  return 1;
}

int orc_dense_grm_bed(const uint8_t* bed, size_t bed_len, int64_t n_fam, int64_t m_tot,
                      const int64_t* sample_idx, int64_t n, double min_maf, double* out,
                      int64_t* n_used) {
  const int64_t bpm = (n_fam + 3) / 4;
  if (bed_len < 3 || (int64_t)bed_len < 3 + bpm * m_tot) return -1;
  if (bed[0] != 0x6C || bed[1] != 0x1B || bed[2] != 0x01) return -1;
  double* z = (double*)malloc(sizeof(double) * (size_t)(m_tot > 0 ? m_tot : 1) * (size_t)n);
  double* d = (double*)malloc(sizeof(double) * (size_t)n);
  int64_t used = 0;
  for (int64_t j = 0; j < m_tot; ++j) {
    double af, mac;
    int64_t nv;
    orc_read_marker(bed, bpm, n_fam, j, sample_idx, n, d);
    orc_compute_af(d, n, &af, &mac, &nv);
    if (af < min_maf || af > 1.0 - min_maf) continue; /* dense.rs:37-39 */
    used += orc_grm_std_marker(d, n, af, z + used * n);
  }
  orc_grm_accumulate(z, n, used, out);
  *n_used = used;
  free(d);
  free(z);
  return 0;
}

void orc_grm_from_dosages(const double* dosages, const double* af, int64_t n, int64_t m,
                          double* out, int64_t* n_used) {
  double* z = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1) * (size_t)n);
  int64_t used = 0;
  for (int64_t j = 0; j < m; ++j) used += orc_grm_std_marker(dosages + j * n, n, af[j], z + used * n);
  orc_grm_accumulate(z, n, used, out);
  *n_used = used;
  free(z);
}

/* ===================================================================== */
/* Synthetic cohorts (no reference counterpart; test and benchmark input) */
/* ===================================================================== */
/* A second statement of the library's seeded generator: every draw is a
 * splitmix64-based hash of (seed, tag, indices); relatives share founder
 * haplotypes (sibling pairs, first-cousin pairs); MCAR missing calls. */
enum { GEN_MAF = 1, GEN_HAP = 2, GEN_REC = 3, GEN_REC2 = 4, GEN_MISS = 5, GEN_COV = 6,
       GEN_EFFECT = 7, GEN_Y = 8, GEN_NOISE = 9 };

static uint64_t gen_mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint64_t gen_hash(uint64_t seed, uint64_t tag, uint64_t a, uint64_t b) {
  uint64_t h = gen_mix(seed ^ (tag * 0xD6E8FEB86659FD93ull));
  h = gen_mix(h ^ (a * 0x9FB21C651E98DF25ull));
  return gen_mix(h + b);
}

static double gen_u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

typedef struct {
  int64_t n, m, n_sib, n_cous, block;
  uint64_t seed;
  double maf_lo, maf_hi, miss;
} gen_layout;

static gen_layout gen_make_layout(const orc_cohort_spec* s) {
  gen_layout L;
  int64_t ns = (int64_t)(s->sib_frac * (double)s->n) / 2 * 2;
  int64_t nc = (int64_t)(s->cousin_frac * (double)s->n) / 2 * 2;
  if (ns < 0) ns = 0;
  if (nc < 0) nc = 0;
  if (ns > s->n / 2 * 2) ns = s->n / 2 * 2;
  if (ns + nc > s->n) nc = (s->n - ns) / 2 * 2;
  L.n = s->n;
  L.m = s->m;
  L.n_sib = ns;
  L.n_cous = nc;
  L.block = s->m > 64 ? (s->m + 63) / 64 : 1;  /* markers per recombination segment */
  L.seed = s->seed;
  L.maf_lo = s->maf_lo;
  L.maf_hi = s->maf_hi;
  L.miss = s->missing_rate;
  return L;
}

static double gen_af(const gen_layout* L, int64_t m) {
  return L->maf_lo + (L->maf_hi - L->maf_lo) * gen_u01(gen_hash(L->seed, GEN_MAF, (uint64_t)m, 0));
}

/* founder haplotype slot (0..7) of the family anchored at sample `base` */
static int gen_hap(const gen_layout* L, int64_t m, double p, int64_t base, int slot) {
  uint64_t f = ((uint64_t)base << 3) | (uint64_t)slot;
  return gen_u01(gen_hash(L->seed, GEN_HAP, (uint64_t)m, f)) < p ? 1 : 0;
}

static int gen_rec(const gen_layout* L, uint64_t tag, uint64_t who, int64_t m) {
  return (int)(gen_hash(L->seed, tag, who, (uint64_t)(m / L->block)) & 1ull);
}

/* alternate-allele count 0..2 of sample i at marker m */
static int gen_genotype(const gen_layout* L, int64_t m, int64_t i, double p) {
  if (i < L->n_sib) {  /* a sibling pair shares parents A (slots 0,1) and B (2,3) */
    int64_t base = i & ~(int64_t)1;
    int a = gen_rec(L, GEN_REC, ((uint64_t)i << 1) | 0u, m);
    int b = gen_rec(L, GEN_REC, ((uint64_t)i << 1) | 1u, m);
    return gen_hap(L, m, p, base, a) + gen_hap(L, m, p, base, 2 + b);
  }
  if (i < L->n_sib + L->n_cous) {  /* cousins: children of two children of G (0,1) x H (2,3) */
    int64_t j = L->n_sib + ((i - L->n_sib) & ~(int64_t)1);
    int c = (int)((i - L->n_sib) & 1);
    int which = gen_rec(L, GEN_REC, ((uint64_t)i << 1) | 0u, m);
    int slot = which == 0
                   ? gen_rec(L, GEN_REC2, ((uint64_t)j << 2) | ((uint64_t)c << 1) | 0u, m)
                   : 2 + gen_rec(L, GEN_REC2, ((uint64_t)j << 2) | ((uint64_t)c << 1) | 1u, m);
    return gen_hap(L, m, p, j, slot) + gen_hap(L, m, p, j, 4 + c);
  }
  return gen_hap(L, m, p, i, 0) + gen_hap(L, m, p, i, 1);
}

static uint32_t gen_code(const gen_layout* L, int64_t m, int64_t i, double p) {
  if (L->miss > 0.0 && gen_u01(gen_hash(L->seed, GEN_MISS, (uint64_t)m, (uint64_t)i)) < L->miss)
    return 1u;  /* 01: missing */
  int g = gen_genotype(L, m, i, p);
  return g == 2 ? 0u : (g == 1 ? 2u : 3u);
}

void orc_gen_bed(const orc_cohort_spec* spec, uint8_t* bed_out) {
  gen_layout L = gen_make_layout(spec);
  const int64_t bpm = (spec->n + 3) / 4;
  bed_out[0] = 0x6C;
  bed_out[1] = 0x1B;
  bed_out[2] = 0x01;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t m = 0; m < spec->m; ++m) {
    const double p = gen_af(&L, m);
    uint8_t* row = bed_out + 3 + m * bpm;
    for (int64_t b = 0; b < bpm; ++b) {
      uint32_t v = 0;
      for (int k = 0; k < 4; ++k) {
        int64_t i = b * 4 + k;
        if (i < L.n) v |= gen_code(&L, m, i, p) << (2 * k);
      }
      row[b] = (uint8_t)v;
    }
  }
}

static double gen_normal(uint64_t h1, uint64_t h2) {  /* Box-Muller, u1 in (0, 1] */
  const double u1 = 1.0 - gen_u01(h1);
  const double u2 = gen_u01(h2);
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

void orc_gen_pheno(const orc_cohort_spec* spec, double* y, double* x) {
  gen_layout L = gen_make_layout(spec);
  const int64_t n = spec->n;
  const int p = 1 + spec->n_covar;
  double beta[64] = {0};
  /* covariates: intercept, N(0,1) (effect 0.3), Bernoulli(0.5) (0.2), then N(0,1) (0.1) */
  for (int64_t i = 0; i < n; ++i) x[i] = 1.0;
  for (int k = 1; k < p; ++k) {
    beta[k] = k == 1 ? 0.3 : (k == 2 ? 0.2 : 0.1);
    for (int64_t i = 0; i < n; ++i) {
      double v;
      if (k == 2) v = gen_u01(gen_hash(L.seed, GEN_COV, (uint64_t)i, (uint64_t)(2 * k))) < 0.5 ? 1.0 : 0.0;
      else v = gen_normal(gen_hash(L.seed, GEN_COV, (uint64_t)i, (uint64_t)(2 * k)),
                          gen_hash(L.seed, GEN_COV, (uint64_t)i, (uint64_t)(2 * k + 1)));
      x[(int64_t)k * n + i] = v;
    }
  }
  /* polygenic score over evenly spaced causal markers (true genotypes), standardised */
  int64_t nc = spec->n_causal > 0 ? spec->n_causal : 500;
  if (nc > spec->m) nc = spec->m;
  if (nc < 1) nc = 1;
  const int64_t stride = spec->m / nc;
  double* pgs = (double*)calloc((size_t)n, sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double acc = 0.0;
    for (int64_t c = 0; c < nc; ++c) {
      const int64_t m = c * stride;
      const double pm = gen_af(&L, m);
      const double sd = sqrt(2.0 * pm * (1.0 - pm));
      const double b = gen_normal(gen_hash(L.seed, GEN_EFFECT, (uint64_t)m, 0),
                                  gen_hash(L.seed, GEN_EFFECT, (uint64_t)m, 1));
      acc += b * ((double)gen_genotype(&L, m, i, pm) - 2.0 * pm) / sd;
    }
    pgs[i] = acc;
  }
  double mean = 0.0, var = 0.0;
  for (int64_t i = 0; i < n; ++i) mean += pgs[i];
  mean /= (double)n;
  for (int64_t i = 0; i < n; ++i) var += (pgs[i] - mean) * (pgs[i] - mean);
  var /= (double)n;
  const double sdv = var > 0 ? sqrt(var) : 1.0;
  for (int64_t i = 0; i < n; ++i) pgs[i] = (pgs[i] - mean) / sdv;
  double* lin = (double*)calloc((size_t)n, sizeof(double));
  for (int64_t i = 0; i < n; ++i) {
    double e = 0.0;
    for (int k = 1; k < p; ++k) e += beta[k] * x[(int64_t)k * n + i];
    lin[i] = e;
  }
  if (spec->trait == 1 /* quantitative */) {
    const double h2 = spec->h2;
    for (int64_t i = 0; i < n; ++i) {
      const double eps = gen_normal(gen_hash(L.seed, GEN_NOISE, (uint64_t)i, 0),
                                    gen_hash(L.seed, GEN_NOISE, (uint64_t)i, 1));
      y[i] = lin[i] + sqrt(h2) * pgs[i] + sqrt(1.0 - h2) * eps;
    }
  } else {
    /* binary: genetic sd on the logistic liability scale for h2, intercept by
     * bisection so that the mean risk equals the prevalence */
    const double h2 = spec->h2 < 0.99 ? spec->h2 : 0.99;
    const double sg = sqrt(h2 * (M_PI * M_PI / 3.0) / (1.0 - h2));
    const double prev = spec->prevalence > 0 && spec->prevalence < 1 ? spec->prevalence : 0.1;
    double lo = -30.0, hi = 30.0;
    for (int it = 0; it < 100; ++it) {
      const double mid = 0.5 * (lo + hi);
      double s = 0.0;
      for (int64_t i = 0; i < n; ++i) s += 1.0 / (1.0 + exp(-(mid + lin[i] + sg * pgs[i])));
      if (s / (double)n < prev) lo = mid;
      else hi = mid;
    }
    const double b0 = 0.5 * (lo + hi);
    for (int64_t i = 0; i < n; ++i) {
      const double mu = 1.0 / (1.0 + exp(-(b0 + lin[i] + sg * pgs[i])));
      y[i] = gen_u01(gen_hash(L.seed, GEN_Y, (uint64_t)i, 0)) < mu ? 1.0 : 0.0;
    }
  }
  free(pgs);
  free(lin);
}
