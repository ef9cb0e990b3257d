"""ctypes access to the CPU oracle (oracle/liboracle.so) — test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use this.
The library is (re)built from oracle/oracle.c with make when missing.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

BINARY, QUANTITATIVE, SURVIVAL = 0, 1, 2
K_IDENTITY, K_OTF, K_EXPLICIT = 0, 1, 2


def _build() -> None:
    src = ORACLE_DIR / "oracle.c"
    if ORACLE_LIB.exists() and ORACLE_LIB.stat().st_mtime >= src.stat().st_mtime:
        return
    subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)


_build()
L = C.CDLL(str(ORACLE_LIB))
P = C.POINTER
_d = P(C.c_double)
_i64 = P(C.c_int64)


class AiRemlConfig(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("tol", C.c_double), ("pcg_tol", C.c_double),
                ("pcg_max_iter", C.c_int), ("n_random_vectors", C.c_int), ("seed", C.c_uint64)]


class AiRemlSummary(C.Structure):
    _fields_ = [("tau", C.c_double * 2), ("iterations", C.c_int), ("converged", C.c_int),
                ("log_likelihood", C.c_double), ("n_kv", C.c_int64), ("pcg_iters", C.c_int64)]


class ChaChaRng(C.Structure):
    _fields_ = [("key", C.c_uint32 * 8), ("counter", C.c_uint64), ("stream", C.c_uint64),
                ("buf", C.c_uint32 * 64), ("idx", C.c_int), ("rounds", C.c_int)]


L.orc_decode_genotype.restype = C.c_double
L.orc_decode_genotype.argtypes = [C.c_uint8, C.c_int]
L.orc_marker_stats.argtypes = [P(C.c_uint8), C.c_size_t, C.c_int64, C.c_int64, _i64, C.c_int64,
                               _d, _d, _i64]
L.orc_chacha_block.argtypes = [P(C.c_uint32), C.c_uint64, C.c_uint64, C.c_int, P(C.c_uint32)]
L.orc_chacha_seed_from_u64.argtypes = [P(ChaChaRng), C.c_uint64, C.c_int]
L.orc_rng_next_u32.restype = C.c_uint32
L.orc_rng_next_u32.argtypes = [P(ChaChaRng)]
L.orc_rng_next_u64.restype = C.c_uint64
L.orc_rng_next_u64.argtypes = [P(ChaChaRng)]
L.orc_rng_gen_range_u64.restype = C.c_uint64
L.orc_rng_gen_range_u64.argtypes = [P(ChaChaRng), C.c_uint64, C.c_uint64]
L.orc_rademacher_probes.argtypes = [C.c_uint64, C.c_int, C.c_int64, _d]
L.orc_select_markers.argtypes = [_d, _d, _i64, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                 C.c_uint64, _i64, _i64, _i64, _i64, _i64]
L.orc_grm_standardize.argtypes = [_d, _d, C.c_int64, C.c_int64, C.c_int, _d]
L.orc_grm_matvec.argtypes = [_d, C.c_int64, C.c_int64, _d, _d, C.c_int]
L.orc_grm_explicit.argtypes = [_d, C.c_int64, C.c_int64, _d]
L.orc_cholesky.argtypes = [_d, C.c_int, _d]
L.orc_chol_solve.argtypes = [_d, C.c_int, _d, _d]
L.orc_pcg_dense.argtypes = [_d, C.c_int, _d, C.c_double, C.c_int, _d, P(C.c_int), _d]
L.orc_fit_glm_irls.argtypes = [_d, _d, C.c_int64, C.c_int, C.c_int, C.c_int, _d]
L.orc_fit_ai_reml.argtypes = [_d, _d, C.c_int64, C.c_int, C.c_int, C.c_int, _d, C.c_int64,
                              C.c_int, P(AiRemlConfig), P(AiRemlSummary), _d, _d, _d, _d, _d]
L.orc_pcg_sigma.argtypes = [_d, C.c_int, _d, C.c_int64, C.c_int64, C.c_int, _d, _d, _d, _d,
                            C.c_double, C.c_int, _d, P(C.c_int), _d, P(C.c_int)]
for f in ("orc_link", "orc_inv_link", "orc_update_mu", "orc_working_weight", "orc_initialize_mu"):
    getattr(L, f).restype = C.c_double
    getattr(L, f).argtypes = [C.c_int, C.c_double]


def dp(a: np.ndarray):
    return a.ctypes.data_as(_d)


def ip(a):
    return None if a is None else a.ctypes.data_as(_i64)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def decode(byte: int, offset: int) -> float:
    return L.orc_decode_genotype(byte, offset)


def marker_stats(bed: np.ndarray, n_fam: int, m_tot: int, sample_idx=None):
    sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
    n = n_fam if sidx is None else sidx.size
    af, mac = np.empty(m_tot), np.empty(m_tot)
    nv = np.empty(m_tot, dtype=np.int64)
    rc = L.orc_marker_stats(bed.ctypes.data_as(P(C.c_uint8)), bed.size, n_fam, m_tot, ip(sidx), n,
                            dp(af), dp(mac), ip(nv))
    if rc != 0:
        raise ValueError("malformed bed")
    return af, mac, nv


def dosages(bed: np.ndarray, n_fam: int, markers, sample_idx=None) -> np.ndarray:
    """m x n dosage matrix (NaN = missing) via plink.rs decode + subset."""
    bpm = (n_fam + 3) // 4
    sidx = np.arange(n_fam) if sample_idx is None else np.asarray(sample_idx)
    markers = np.asarray(markers)
    rows = bed[3:].reshape(-1, bpm)[markers]  # (m, bpm)
    codes = (rows[:, sidx // 4] >> (2 * (sidx % 4)).astype(np.uint8)) & 3
    lut = np.array([2.0, np.nan, 1.0, 0.0])
    return lut[codes]


def chacha_block(key_words, counter: int, stream: int, rounds: int) -> np.ndarray:
    k = (C.c_uint32 * 8)(*[int(x) for x in key_words])
    out = (C.c_uint32 * 16)()
    L.orc_chacha_block(k, counter, stream, rounds, out)
    return np.array(out, dtype=np.uint32)


def chacha8_u32_stream(seed: int, count: int) -> np.ndarray:
    r = ChaChaRng()
    L.orc_chacha_seed_from_u64(C.byref(r), seed, 8)
    return np.array([L.orc_rng_next_u32(C.byref(r)) for _ in range(count)], dtype=np.uint32)


def gen_range_u64(seed: int, low: int, high: int, count: int) -> np.ndarray:
    r = ChaChaRng()
    L.orc_chacha_seed_from_u64(C.byref(r), seed, 8)
    return np.array([L.orc_rng_gen_range_u64(C.byref(r), low, high) for _ in range(count)],
                    dtype=np.uint64)


def probes(seed: int, n_vec: int, n: int) -> np.ndarray:
    out = np.empty((n_vec, n))
    L.orc_rademacher_probes(seed, n_vec, n, dp(out))
    return out


def select_markers(af, mac, nv, n, min_maf=0.01, max_missing=0.15, seed=12345):
    af, mac = f64(af), f64(mac)
    nv = np.ascontiguousarray(nv, dtype=np.int64)
    m = af.size
    g = np.empty(max(m, 1), dtype=np.int64)
    v = np.empty(max(m, 1), dtype=np.int64)
    mg, mv, npass = C.c_int64(), C.c_int64(), C.c_int64()
    rc = L.orc_select_markers(dp(af), dp(mac), ip(nv), m, n, min_maf, max_missing, seed, ip(g),
                              C.byref(mg), ip(v), C.byref(mv), C.byref(npass))
    if rc != 0:
        raise ValueError("no marker passes QC")
    return g[: mg.value].copy(), v[: mv.value].copy()


def standardize(dos: np.ndarray, af, mode: int) -> np.ndarray:
    dos = f64(dos)
    m, n = dos.shape
    z = np.empty_like(dos)
    L.orc_grm_standardize(dp(dos), dp(f64(af)), n, m, mode, dp(z))
    return z


def grm_matvec(z: np.ndarray, v, mode: int) -> np.ndarray:
    m, n = z.shape
    out = np.empty(n)
    L.orc_grm_matvec(dp(f64(z)), n, m, dp(f64(v)), dp(out), mode)
    return out


def grm_explicit(z: np.ndarray) -> np.ndarray:
    m, n = z.shape
    k = np.empty((n, n))
    L.orc_grm_explicit(dp(f64(z)), n, m, dp(k))
    return k


def cholesky(a: np.ndarray):
    a = f64(a)
    p = a.shape[0]
    l = np.empty_like(a)
    rc = L.orc_cholesky(dp(a), p, dp(l))
    return (None if rc != 0 else l)


def chol_solve(l: np.ndarray, b) -> np.ndarray:
    p = l.shape[0]
    x = np.empty(p)
    L.orc_chol_solve(dp(f64(l)), p, dp(f64(b)), dp(x))
    return x


def pcg_dense(a: np.ndarray, b, tol=1e-5, max_iter=500):
    a = f64(a)
    n = a.shape[0]
    x = np.empty(n)
    it = C.c_int()
    rs = C.c_double()
    conv = L.orc_pcg_dense(dp(a), n, dp(f64(b)), tol, max_iter, dp(x), C.byref(it), C.byref(rs))
    return x, it.value, rs.value, bool(conv)


def pcg_sigma(kind, grm, n, m, kmode, w, tau, b, x0=None, tol=1e-5, max_iter=500):
    x = np.empty(n)
    it, cv = C.c_int(), C.c_int()
    rs = C.c_double()
    g = None if grm is None else dp(f64(grm))
    L.orc_pcg_sigma(None, kind, g, n, m, kmode, dp(f64(w)), dp(f64(tau)), dp(f64(b)),
                    None if x0 is None else dp(f64(x0)), tol, max_iter, dp(x), C.byref(it),
                    C.byref(rs), C.byref(cv))
    return x, it.value, rs.value, bool(cv.value)


def fit_glm_irls(y, x: np.ndarray, trait: int, max_iter=25) -> np.ndarray:
    n, p = x.shape
    xc = np.asfortranarray(x).ravel(order="F").copy()
    a = np.empty(p)
    rc = L.orc_fit_glm_irls(dp(f64(y)), dp(xc), n, p, trait, max_iter, dp(a))
    if rc != 0:
        raise ValueError("IRLS Cholesky failed")
    return a


def fit_ai_reml(y, x: np.ndarray, trait: int, kind: int, grm, m: int = 0, kmode: int = 0,
                max_iter=30, tol=0.02, pcg_tol=1e-5, pcg_max_iter=500, n_random_vectors=30,
                seed=12345):
    n, p = x.shape
    xc = np.asfortranarray(x).ravel(order="F").copy()
    cfg = AiRemlConfig(max_iter, tol, pcg_tol, pcg_max_iter, n_random_vectors, seed)
    out = AiRemlSummary()
    trace = np.full(2 * max(max_iter, 1), np.nan)
    alpha, mu, eta, w = np.empty(p), np.empty(n), np.empty(n), np.empty(n)
    g = None if grm is None else dp(f64(grm))
    rc = L.orc_fit_ai_reml(dp(f64(y)), dp(xc), n, p, trait, kind, g, m, kmode, C.byref(cfg),
                           C.byref(out), dp(trace), dp(alpha), dp(mu), dp(eta), dp(w))
    if rc != 0:
        raise ValueError(f"oracle fit_ai_reml failed ({rc})")
    it = out.iterations
    return dict(tau=np.array(out.tau[:]), iterations=it, converged=bool(out.converged),
                log_likelihood=out.log_likelihood, n_kv=out.n_kv, pcg_iters=out.pcg_iters,
                tau_trace=trace[: 2 * it].reshape(-1, 2), alpha=alpha, mu=mu, eta=eta, w=w)


# ---------------------------------------------------------------- variance ratio
class VrConfig(C.Structure):
    _fields_ = [("n_markers", C.c_int), ("min_mac", C.c_double), ("ratio_cv_cutoff", C.c_double),
                ("seed", C.c_uint64), ("use_categorical", C.c_int), ("xadjust", C.c_int)]


class VrSummary(C.Structure):
    _fields_ = [("variance_ratio", C.c_double), ("n_markers_used", C.c_int),
                ("n_categories", C.c_int), ("cat_upper", C.c_double * 8),
                ("cat_vr", C.c_double * 8), ("n_kv", C.c_int64)]


L.orc_rng_gen_range_u32.restype = C.c_uint32
L.orc_rng_gen_range_u32.argtypes = [P(ChaChaRng), C.c_uint32, C.c_uint32]
L.orc_shuffled_indices.argtypes = [C.c_uint64, C.c_int64, _i64]
L.orc_variance_ratio.restype = C.c_int
L.orc_variance_ratio.argtypes = [_d, _d, C.c_int64, _d, _d, _d, C.c_int, _d, C.c_int64, C.c_int,
                                 C.c_int, _d, C.c_int64, C.c_int, P(VrConfig), P(VrSummary), _d,
                                 _i64]


def shuffled_indices(seed: int, length: int) -> np.ndarray:
    out = np.empty(max(length, 1), dtype=np.int64)
    L.orc_shuffled_indices(seed, length, out.ctypes.data_as(_i64))
    return out[:length]


def variance_ratio(dosages, mac, mu, w, tau, trait: int, x: np.ndarray, kind: int, grm,
                   m: int = 0, kmode: int = 0, n_markers=30, min_mac=20.0, cutoff=0.001,
                   seed=12345, categorical=False, xadjust=0):
    d = np.ascontiguousarray(dosages, dtype=np.float64)
    n_cand, n = d.shape
    p = x.shape[1]
    xc = np.asfortranarray(x).ravel(order="F").copy()
    cfg = VrConfig(n_markers, min_mac, cutoff, seed, int(categorical), xadjust)
    out = VrSummary()
    vr = np.empty(max(n_cand, 1))
    used = np.empty(max(n_cand, 1), dtype=np.int64)
    g = None if grm is None else dp(f64(grm))
    rc = L.orc_variance_ratio(dp(d), dp(f64(mac)), n_cand, dp(f64(mu)), dp(f64(w)),
                              dp(f64(tau)), trait, dp(xc), n, p, kind, g, m, kmode,
                              C.byref(cfg), C.byref(out), dp(vr), used.ctypes.data_as(_i64))
    k = out.n_markers_used
    return dict(rc=rc, variance_ratio=out.variance_ratio, n_used=k, per_marker=vr[:k].copy(),
                used=used[:k].copy(), n_kv=out.n_kv,
                categorical=[(out.cat_upper[i], out.cat_vr[i]) for i in range(out.n_categories)])


# ---- explicit GRM (saige-core/src/grm/dense.rs, grm/sparse.rs) -------------
L.orc_dense_grm_bed.argtypes = [P(C.c_uint8), C.c_size_t, C.c_int64, C.c_int64, _i64, C.c_int64,
                                C.c_double, _d, _i64]
L.orc_grm_from_dosages.argtypes = [_d, _d, C.c_int64, C.c_int64, _d, _i64]


def dense_grm_bed(bed: np.ndarray, n_fam: int, m_tot: int, min_maf=0.01, sample_idx=None):
    """compute_dense_grm (dense.rs:22-112): (K n x n, n_markers_used)."""
    sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
    n = n_fam if sidx is None else sidx.size
    out = np.empty((n, n))
    used = np.zeros(1, dtype=np.int64)
    rc = L.orc_dense_grm_bed(bed.ctypes.data_as(P(C.c_uint8)), bed.size, n_fam, m_tot, ip(sidx), n,
                             min_maf, dp(out), ip(used))
    if rc != 0:
        raise ValueError("malformed bed")
    return out, int(used[0])


def grm_from_dosages(dos: np.ndarray, af):
    """compute_grm_from_dosages (dense.rs:115-186); m == 0 gives a 0 x 0 matrix."""
    dos = f64(dos)
    m, n = dos.shape
    if m == 0:
        return np.zeros((0, 0)), 0
    out = np.empty((n, n))
    used = np.zeros(1, dtype=np.int64)
    L.orc_grm_from_dosages(dp(dos), dp(f64(af)), n, m, dp(out), ip(used))
    return out, int(used[0])


def sparse_from_dense(k: np.ndarray, cutoff: float):
    """sparse.rs:36-53 thresholding, stored as the writer lists it
    (sparse_grm_io.rs:92-107): upper triangle with the diagonal, row-major,
    (rows, cols, vals) 0-based."""
    n = k.shape[0]
    iu, ju = np.triu_indices(n)
    v = k[iu, ju]
    keep = (iu == ju) | (np.abs(v) >= cutoff)
    return iu[keep].astype(np.int32), ju[keep].astype(np.int32), v[keep]


def sparse_grm_text(n: int, rows, cols, vals) -> str:
    """The .sparseGRM.mtx text write_sparse_grm produces (sparse_grm_io.rs:73-115);
    Rust's {:.10} and C's %.10f both print the exact decimal value rounded."""
    lines = ["%%MatrixMarket matrix coordinate real symmetric", f"{n} {n} {len(vals)}"]
    lines += ["%d %d %.10f" % (i + 1, j + 1, v) for i, j, v in zip(rows, cols, vals)]
    return "\n".join(lines) + "\n"


def gen_f64(rng: ChaChaRng) -> float:
    """rand 0.8 Standard for f64: the top 53 bits of next_u64, times 2^-53."""
    return (L.orc_rng_next_u64(C.byref(rng)) >> 11) * (1.0 / (1 << 53))


def chacha8(seed: int) -> ChaChaRng:
    r = ChaChaRng()
    L.orc_chacha_seed_from_u64(C.byref(r), seed, 8)
    return r


# ---- synthetic cohorts (the library's generator, restated) ------------------
class CohortSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("n", C.c_int64), ("m", C.c_int64),
                ("sib_frac", C.c_double), ("cousin_frac", C.c_double),
                ("missing_rate", C.c_double), ("maf_lo", C.c_double), ("maf_hi", C.c_double),
                ("trait", C.c_int32), ("n_covar", C.c_int32), ("prevalence", C.c_double),
                ("h2", C.c_double), ("n_causal", C.c_int32), ("reserved", C.c_int32)]


L.orc_gen_bed.argtypes = [P(CohortSpec), P(C.c_uint8)]
L.orc_gen_pheno.argtypes = [P(CohortSpec), _d, _d]


def cohort_spec(seed=12345, n=2000, m=5000, sib_frac=0.10, cousin_frac=0.0, missing_rate=0.01,
                maf_lo=0.01, maf_hi=0.5, trait=BINARY, n_covar=2, prevalence=0.10, h2=0.2,
                n_causal=500) -> CohortSpec:
    return CohortSpec(seed, n, m, sib_frac, cousin_frac, missing_rate, maf_lo, maf_hi, trait,
                      n_covar, prevalence, h2, n_causal, 0)


def gen_bed(spec: CohortSpec) -> np.ndarray:
    out = np.empty(3 + spec.m * ((spec.n + 3) // 4), dtype=np.uint8)
    L.orc_gen_bed(C.byref(spec), out.ctypes.data_as(P(C.c_uint8)))
    return out


def gen_pheno(spec: CohortSpec):
    y = np.empty(spec.n)
    x = np.empty(spec.n * (1 + spec.n_covar))
    L.orc_gen_pheno(C.byref(spec), dp(y), dp(x))
    return y, x.reshape(1 + spec.n_covar, spec.n).T


L.orc_grm_matmul_f64_packed.restype = C.c_int
L.orc_grm_matmul_f64_packed.argtypes = [P(C.c_uint8), C.c_int64, C.c_int64, _i64, C.c_int64, _d,
                                        _d, C.c_int, _d]


def grm_matmul_f64_packed(bed: np.ndarray, n: int, rows, af, v: np.ndarray) -> np.ndarray:
    """FP64 K V on the packed .bed rows `rows` (all n samples in file order); v is
    (nrhs, n) or (n,); af per row."""
    vv = np.ascontiguousarray(np.atleast_2d(v), dtype=np.float64)
    assert vv.shape[0] <= 64
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.empty_like(vv)
    body = np.ascontiguousarray(bed[3:])
    L.orc_grm_matmul_f64_packed(body.ctypes.data_as(P(C.c_uint8)), (n + 3) // 4, n, ip(rows),
                                rows.size, dp(f64(af)), dp(vv), vv.shape[0], dp(out))
    return out if np.ndim(v) == 2 else out[0]
