// Seeded synthetic cohorts: genotypes with sibling and first-cousin
// relatedness, MCAR missing calls, covariates and a polygenic phenotype.
// Every draw is a counter-based hash of (seed, tag, indices), so any subset
// of the genotype matrix can be produced independently, on the host or on
// the device, with identical results.
#pragma once
#include <stdint.h>

#include "../../include/saige_gpu.h"

#ifdef __CUDACC__
#define SG_HD __host__ __device__ __forceinline__
#else
#define SG_HD inline
#endif

namespace saige {
namespace cohort {

enum : uint64_t {
  kTagMaf = 1,
  kTagHap = 2,
  kTagRec = 3,
  kTagRec2 = 4,
  kTagMiss = 5,
  kTagCov = 6,
  kTagEffect = 7,
  kTagY = 8,
  kTagNoise = 9,
};

// splitmix64 finaliser (Steele, Lea, Flood 2014).
SG_HD uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

SG_HD uint64_t hash4(uint64_t seed, uint64_t tag, uint64_t a, uint64_t b) {
  uint64_t h = mix64(seed ^ (tag * 0xD6E8FEB86659FD93ull));
  h = mix64(h ^ (a * 0x9FB21C651E98DF25ull));
  return mix64(h + b);
}

SG_HD double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

struct Layout {
  int64_t n, m;
  int64_t n_sib;   // samples [0, n_sib) form sibling pairs
  int64_t n_cous;  // samples [n_sib, n_sib + n_cous) form first-cousin pairs
  int64_t block;   // markers per recombination segment
  uint64_t seed;
  double maf_lo, maf_hi, miss;
};

inline Layout make_layout(const saige_cohort_spec& s) {
  Layout L;
  L.n = s.n;
  L.m = s.m;
  int64_t ns = (int64_t)(s.sib_frac * (double)s.n) / 2 * 2;
  int64_t nc = (int64_t)(s.cousin_frac * (double)s.n) / 2 * 2;
  if (ns < 0) ns = 0;
  if (nc < 0) nc = 0;
  if (ns > s.n / 2 * 2) ns = s.n / 2 * 2;
  if (ns + nc > s.n) nc = (s.n - ns) / 2 * 2;
  L.n_sib = ns;
  L.n_cous = nc;
  L.block = s.m > 64 ? (s.m + 63) / 64 : 1;
  L.seed = s.seed;
  L.maf_lo = s.maf_lo;
  L.maf_hi = s.maf_hi;
  L.miss = s.missing_rate;
  return L;
}

SG_HD double allele_freq(const Layout& L, int64_t m) {
  return L.maf_lo + (L.maf_hi - L.maf_lo) * u01(hash4(L.seed, kTagMaf, (uint64_t)m, 0));
}

// Founder haplotype: slot s (0..7) of the family anchored at sample `base`.
SG_HD int hap_allele(const Layout& L, int64_t m, double p, int64_t base, int slot) {
  uint64_t f = ((uint64_t)base << 3) | (uint64_t)slot;
  return u01(hash4(L.seed, kTagHap, (uint64_t)m, f)) < p ? 1 : 0;
}

SG_HD int rec_bit(const Layout& L, uint64_t tag, uint64_t who, int64_t m) {
  return (int)(hash4(L.seed, tag, who, (uint64_t)(m / L.block)) & 1ull);
}

// True alt-allele count (0..2) of sample i at marker m, before missingness.
SG_HD int true_genotype(const Layout& L, int64_t m, int64_t i, double p) {
  if (i < L.n_sib) {
    // Parents A (slots 0,1) and B (slots 2,3) shared by the pair.
    int64_t base = i & ~(int64_t)1;
    int a = rec_bit(L, kTagRec, ((uint64_t)i << 1) | 0u, m);
    int b = rec_bit(L, kTagRec, ((uint64_t)i << 1) | 1u, m);
    return hap_allele(L, m, p, base, a) + hap_allele(L, m, p, base, 2 + b);
  }
  if (i < L.n_sib + L.n_cous) {
    // Grandparents G (0,1) and H (2,3); parent c is their child; the cousin
    // takes one haplotype of its parent and one of an unrelated spouse.
    int64_t j = L.n_sib + ((i - L.n_sib) & ~(int64_t)1);
    int c = (int)((i - L.n_sib) & 1);
    int which = rec_bit(L, kTagRec, ((uint64_t)i << 1) | 0u, m);  // parent hap 0 or 1
    int slot;
    if (which == 0) slot = rec_bit(L, kTagRec2, ((uint64_t)j << 2) | ((uint64_t)c << 1) | 0u, m);
    else slot = 2 + rec_bit(L, kTagRec2, ((uint64_t)j << 2) | ((uint64_t)c << 1) | 1u, m);
    return hap_allele(L, m, p, j, slot) + hap_allele(L, m, p, j, 4 + c);
  }
  return hap_allele(L, m, p, i, 0) + hap_allele(L, m, p, i, 1);
}

SG_HD bool is_missing(const Layout& L, int64_t m, int64_t i) {
  return L.miss > 0.0 && u01(hash4(L.seed, kTagMiss, (uint64_t)m, (uint64_t)i)) < L.miss;
}

// PLINK 2-bit code of (m, i): 00 = 2 copies of A1, 10 = 1, 11 = 0, 01 = missing.
SG_HD uint32_t bed_code(const Layout& L, int64_t m, int64_t i, double p) {
  if (is_missing(L, m, i)) return 1u;
  int g = true_genotype(L, m, i, p);
  return g == 2 ? 0u : (g == 1 ? 2u : 3u);
}

// One byte of marker m's row: samples 4*byte .. 4*byte+3 (padding codes 00,
// as PLINK writes them).
SG_HD uint8_t bed_byte(const Layout& L, int64_t m, int64_t byte, double p) {
  uint32_t v = 0;
  for (int k = 0; k < 4; ++k) {
    int64_t i = byte * 4 + k;
    if (i < L.n) v |= bed_code(L, m, i, p) << (2 * k);
  }
  return (uint8_t)v;
}

}  // namespace cohort
}  // namespace saige
