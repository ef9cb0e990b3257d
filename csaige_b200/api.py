"""Host-side mirror of the saige-rs fit-null API over the sm_100a library.

Names, argument meaning and error behaviour follow the saige-rs types they
stand in for (paths relative to the frhl/CSAIGE tree):

  OnTheFlyGrm         saige-core/src/glmm/pcg.rs:91-180
  PcgSolver/PcgResult saige-linalg/src/decomposition.rs:167-298
  solve_mixed_model_pcg, SaigePcgConfig   saige-core/src/glmm/pcg.rs:12-78
  AiRemlConfig, AiRemlResult, fit_ai_reml saige-core/src/glmm/ai_reml.rs:20-427
  TraitType           saige-core/src/glmm/link.rs:7-12
  bed_marker_stats    saige-geno/src/plink.rs:237-267 + traits.rs:42-54
  select_grm_markers  saige-cli/src/commands/fit_null.rs:209-259

Every call goes through the C ABI of libsaige_gpu.so; nothing is computed in
Python.  Where the reference panics (assert_eq! on dimensions) this module
raises SaigeError(SAIGE_EINVAL).
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import LIB, SaigeError, check

PREC_FP32 = _lib.PREC_FP32
PREC_MIXED = _lib.PREC_MIXED
SOLVE_SINGLE = _lib.SOLVE_SINGLE
SOLVE_BLOCK = _lib.SOLVE_BLOCK
WARM_ZERO = _lib.WARM_ZERO
WARM_PREVIOUS = _lib.WARM_PREVIOUS
WARM_LEARNED = _lib.WARM_LEARNED
WARM_RECYCLED = _lib.WARM_RECYCLED
PRECOND_UNIT = 0    # 1 / (tau0 / w + tau1): diag K taken as 1 (ai_reml.rs:142-164)
PRECOND_DIAG_K = 1  # 1 / (tau0 / w + tau1 K_ii) with the exact diagonal


class TraitType(enum.IntEnum):
    Binary = _lib.TRAIT_BINARY
    Quantitative = _lib.TRAIT_QUANTITATIVE
    Survival = _lib.TRAIT_SURVIVAL


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int64))


def _f64(a, n: Optional[int] = None) -> np.ndarray:
    out = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if n is not None and out.size != n:
        raise SaigeError(_lib.EINVAL, f"expected {n} values, got {out.size}")
    return out


def device_count() -> int:
    return int(LIB.saige_device_count())


def version() -> int:
    return int(LIB.saige_version())


# ---------------------------------------------------------------------------
# genotype input
# ---------------------------------------------------------------------------
def _bed_array(bed) -> np.ndarray:
    if isinstance(bed, (bytes, bytearray, memoryview)):
        return np.frombuffer(bed, dtype=np.uint8)
    return np.ascontiguousarray(np.asarray(bed, dtype=np.uint8))


def bed_marker_stats(bed, n_fam: int, m_tot: int, sample_idx: Optional[Sequence[int]] = None):
    """(af, mac, n_valid) per marker over the sample subset, integer-exact on the GPU."""
    b = _bed_array(bed)
    sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
    n = n_fam if sidx is None else sidx.size
    af = np.empty(m_tot)
    mac = np.empty(m_tot)
    nv = np.empty(m_tot, dtype=np.int64)
    check(
        LIB.saige_bed_marker_stats(
            b.ctypes.data_as(C.POINTER(C.c_uint8)), b.size, n_fam, m_tot, _i64ptr(sidx), n,
            _dptr(af), _dptr(mac), _i64ptr(nv)
        )
    )
    return af, mac, nv


def bed_marker_stats_dev(bed_ptr: int, bed_len: int, n_fam: int, m_tot: int,
                         sample_idx: Optional[Sequence[int]] = None):
    """bed_marker_stats for a .bed already in device memory (bed_ptr: device address)."""
    sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
    n = n_fam if sidx is None else sidx.size
    af = np.empty(m_tot)
    mac = np.empty(m_tot)
    nv = np.empty(m_tot, dtype=np.int64)
    check(LIB.saige_bed_marker_stats_dev(C.c_void_p(bed_ptr), bed_len, n_fam, m_tot, _i64ptr(sidx),
                                         n, _dptr(af), _dptr(mac), _i64ptr(nv)))
    return af, mac, nv


def release_cached_memory() -> None:
    """Frees the library's cached large device blocks (see saige_release_cached_memory)."""
    check(LIB.saige_release_cached_memory())


def rademacher_probes(seed: int, n_vec: int, n: int, device: int = -1) -> np.ndarray:
    """The +1/-1 probe vectors of fit_ai_reml (ai_reml.rs:121-130), shape (n_vec, n),
    generated on the GPU from the ChaCha8Rng::seed_from_u64(seed) stream."""
    out = np.empty((n_vec, n))
    check(LIB.saige_rademacher_probes(seed, n_vec, n, _dptr(out), device))
    return out


def select_grm_markers(af, mac, n_valid, n: int, min_maf: float = 0.01,
                       max_missing: float = 0.15, seed: int = 12345):
    """(grm_idx, vr_idx): QC plus the variance-ratio marker split of fit-null."""
    af = _f64(af)
    mac = _f64(mac, af.size)
    nv = np.ascontiguousarray(n_valid, dtype=np.int64)
    m = af.size
    g = np.empty(max(m, 1), dtype=np.int64)
    v = np.empty(max(m, 1), dtype=np.int64)
    mg = C.c_int64()
    mv = C.c_int64()
    check(
        LIB.saige_select_grm_markers(
            _dptr(af), _dptr(mac), _i64ptr(nv), m, n, min_maf, max_missing, seed, _i64ptr(g),
            C.byref(mg), _i64ptr(v), C.byref(mv)
        )
    )
    return g[: mg.value].copy(), v[: mv.value].copy()


# ---------------------------------------------------------------------------
# GRM operator
# ---------------------------------------------------------------------------
class OnTheFlyGrm:
    """K v = Z (Z' v) / M over 2-bit genotypes resident in HBM."""

    def __init__(self, handle: C.c_void_p, precision: int = PREC_FP32):
        self._h = handle
        n = C.c_int64()
        m = C.c_int64()
        check(LIB.saige_grm_dims(self._h, C.byref(n), C.byref(m)))
        self.n_samples = n.value
        self.n_markers = m.value
        self.precision = precision

    @classmethod
    def new(cls, dosages, allele_freqs, device: int = -1, precision: int = PREC_FP32):
        """OnTheFlyGrm::new(dosages, allele_freqs): m dosage vectors of n hard calls."""
        d = np.asarray(dosages, dtype=np.float64)
        if d.ndim != 2:
            raise SaigeError(_lib.EINVAL, "dosages must be m x n")
        m, n = d.shape
        d = np.ascontiguousarray(d)
        af = _f64(allele_freqs, m)
        h = C.c_void_p()
        check(LIB.saige_grm_create_from_dosages(_dptr(d), n, m, _dptr(af), device, C.byref(h)))
        return cls(h, precision)

    @classmethod
    def from_bed(cls, bed, n_fam: int, m_tot: int, marker_idx, allele_freqs,
                 sample_idx: Optional[Sequence[int]] = None, device: int = -1,
                 precision: int = PREC_FP32):
        b = _bed_array(bed)
        midx = np.ascontiguousarray(marker_idx, dtype=np.int64)
        af = _f64(allele_freqs, midx.size)
        sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
        n = n_fam if sidx is None else sidx.size
        h = C.c_void_p()
        check(
            LIB.saige_grm_create_from_bed(
                b.ctypes.data_as(C.POINTER(C.c_uint8)), b.size, n_fam, m_tot, _i64ptr(sidx), n,
                _i64ptr(midx), midx.size, _dptr(af), device, C.byref(h)
            )
        )
        return cls(h, precision)

    @classmethod
    def from_bed_dev(cls, bed_ptr: int, bed_len: int, n_fam: int, m_tot: int, marker_idx,
                     allele_freqs, sample_idx=None, device: int = -1,
                     precision: int = PREC_FP32):
        midx = np.ascontiguousarray(marker_idx, dtype=np.int64)
        af = _f64(allele_freqs, midx.size)
        sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
        n = n_fam if sidx is None else sidx.size
        h = C.c_void_p()
        check(
            LIB.saige_grm_create_from_bed_dev(
                C.c_void_p(bed_ptr), bed_len, n_fam, m_tot, _i64ptr(sidx), n, _i64ptr(midx),
                midx.size, _dptr(af), device, C.byref(h)
            )
        )
        return cls(h, precision)

    def close(self) -> None:
        if getattr(self, "_h", None):
            LIB.saige_grm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mat_vec(self, v, precision: Optional[int] = None) -> np.ndarray:
        """K v for one vector (n,) or a block (nrhs, n)."""
        a = _f64(v)
        one = a.ndim == 1
        a = a.reshape(1, -1) if one else a
        if a.shape[1] != self.n_samples:
            raise SaigeError(_lib.EINVAL, f"v.len() = {a.shape[1]} != n_samples = {self.n_samples}")
        out = np.empty_like(a)
        prec = self.precision if precision is None else precision
        check(LIB.saige_grm_matvec(self._h, _dptr(a), _dptr(out), self.n_samples, a.shape[0], prec))
        return out[0] if one else out

    def mat_vec_dev(self, v_ptr: int, out_ptr: int, nrhs: int = 1,
                    precision: Optional[int] = None, stream: int = 0) -> None:
        prec = self.precision if precision is None else precision
        check(LIB.saige_grm_matvec_dev(self._h, C.c_void_p(v_ptr), C.c_void_p(out_ptr),
                                       self.n_samples, nrhs, prec, C.c_void_p(stream or None)))

    def diag(self) -> np.ndarray:
        """K_ii = (1/M) sum_m z_im^2 in FP64 (Get_Diagof_StdGeno,
        src/SAIGE_fitGLMM_fast.cpp:642-680)."""
        out = np.empty(self.n_samples)
        check(LIB.saige_grm_diag(self._h, _dptr(out), self.n_samples))
        return out

    def __call__(self, v):
        return self.mat_vec(v)


# ---------------------------------------------------------------------------
# PCG
# ---------------------------------------------------------------------------
@dataclass
class PcgResult:
    x: np.ndarray
    iterations: int
    residual: float
    converged: bool


class PcgSolver:
    """PcgSolver { tol, max_iter } on the fit-null operator of a GRM handle."""

    def __init__(self, tol: float = 1e-5, max_iter: int = 500):
        self.tol = tol
        self.max_iter = max_iter

    def solve(self, grm: OnTheFlyGrm, w, tau, b, x0=None, precision: Optional[int] = None):
        """Solve (tau0 W^-1 + tau1 K) x = b; b is (n,) or a block (nrhs, n).

        A block returns one PcgResult per column."""
        n = grm.n_samples
        bb = _f64(b)
        one = bb.ndim == 1
        bb = bb.reshape(1, -1) if one else bb
        q = bb.shape[0]
        if bb.shape[1] != n:
            raise SaigeError(_lib.EINVAL, "b has the wrong length")
        wv = _f64(w, n)
        t = _f64(tau, 2)
        xx = np.empty_like(bb)
        x0a = None if x0 is None else _f64(x0, q * n).reshape(q, n)
        it = np.zeros(q, dtype=np.int32)
        rs = np.zeros(q)
        cv = np.zeros(q, dtype=np.uint8)
        opt = _lib.PcgOptions(self.tol, self.max_iter,
                              grm.precision if precision is None else precision)
        check(LIB.saige_pcg_solve(grm._h, _dptr(wv), _dptr(t), _dptr(bb),
                                  None if x0a is None else _dptr(x0a), _dptr(xx), n, q,
                                  C.byref(opt), it.ctypes.data_as(C.POINTER(C.c_int32)),
                                  _dptr(rs), cv.ctypes.data_as(C.POINTER(C.c_uint8))))
        res = [PcgResult(xx[c].copy(), int(it[c]), float(rs[c]), bool(cv[c])) for c in range(q)]
        return res[0] if one else res


@dataclass
class SaigePcgConfig:
    tol: float = 1e-5
    max_iter: int = 500


def solve_mixed_model_pcg(tau, w, grm: OnTheFlyGrm, b, config: SaigePcgConfig = SaigePcgConfig(),
                          precision: Optional[int] = None) -> PcgResult:
    """(tau_e W + tau_g GRM) x = b, the score-test convention of pcg.rs:37-78."""
    n = grm.n_samples
    bb = _f64(b, n)
    wv = _f64(w, n)
    t = _f64(tau, 2)
    x = np.empty(n)
    it = C.c_int32()
    rs = C.c_double()
    cv = C.c_uint8()
    opt = _lib.PcgOptions(config.tol, config.max_iter,
                          grm.precision if precision is None else precision)
    check(LIB.saige_solve_mixed_model_pcg(grm._h, _dptr(t), _dptr(wv), _dptr(bb), _dptr(x), n,
                                          C.byref(opt), C.byref(it), C.byref(rs), C.byref(cv)))
    return PcgResult(x, it.value, rs.value, bool(cv.value))


# ---------------------------------------------------------------------------
# AI-REML
# ---------------------------------------------------------------------------
@dataclass
class AiRemlConfig:
    max_iter: int = 30
    tol: float = 0.02
    pcg_tol: float = 1e-5
    pcg_max_iter: int = 500
    n_random_vectors: int = 30
    use_sparse_grm: bool = False  # parsed by the reference, never read (ai_reml.rs:33)
    seed: int = 12345
    precision: int = PREC_FP32
    solve: int = SOLVE_SINGLE
    warm_start: int = WARM_ZERO
    precond: int = PRECOND_UNIT


@dataclass
class AiRemlResult:
    tau: np.ndarray
    iterations: int
    converged: bool
    mu: np.ndarray
    working_weights: np.ndarray
    residuals: np.ndarray
    eta: np.ndarray
    alpha: np.ndarray
    log_likelihood: float
    n_kv: int = 0
    n_kv_launches: int = 0
    pcg_iters: int = 0
    seconds: float = 0.0
    tau_trace: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))
    learned_trainings: int = 0
    learned_uses: int = 0
    learned_r2: float = 0.0
    learned_seconds: float = 0.0


def _design(x, n: int) -> tuple[np.ndarray, int]:
    a = np.asarray(x, dtype=np.float64)
    if a.ndim == 1:
        a = a.reshape(n, -1, order="F")
    if a.shape[0] != n:
        raise SaigeError(_lib.EINVAL, f"x.nrows() = {a.shape[0]} != n = {n}")
    # column-major n x p, copied only when the layout differs (the library reads it)
    return np.asfortranarray(a).ravel(order="F"), a.shape[1]


def fit_ai_reml(y, x, grm: OnTheFlyGrm, trait_type: TraitType,
                config: AiRemlConfig = AiRemlConfig()) -> AiRemlResult:
    """fit_ai_reml(y, x, |v| grm.mat_vec(v), trait_type, config).  x is n x p."""
    yy = _f64(y)
    n = yy.size
    if n != grm.n_samples:
        raise SaigeError(_lib.EINVAL, "y.len() != n_samples")
    xc, p = _design(x, n)
    cfg = _lib.AiRemlConfigC(config.max_iter, config.tol, config.pcg_tol, config.pcg_max_iter,
                             config.n_random_vectors, config.seed, config.precision, config.solve,
                             config.warm_start, config.precond)
    out = _lib.AiRemlSummaryC()
    alpha = np.zeros(p)
    mu = np.zeros(n)
    eta = np.zeros(n)
    w = np.zeros(n)
    trace = np.full(2 * max(config.max_iter, 1), np.nan)
    check(LIB.saige_fit_ai_reml(grm._h, _dptr(yy), _dptr(xc), n, p, int(trait_type),
                                C.byref(cfg), C.byref(out), _dptr(alpha), _dptr(mu), _dptr(eta),
                                _dptr(w), _dptr(trace)))
    it = out.iterations
    return AiRemlResult(
        tau=np.array([out.tau[0], out.tau[1]]), iterations=it, converged=bool(out.converged),
        mu=mu, working_weights=w, residuals=yy - mu, eta=eta, alpha=alpha,
        log_likelihood=out.log_likelihood, n_kv=out.n_kv, n_kv_launches=out.n_kv_launches,
        pcg_iters=out.pcg_iters, seconds=out.seconds,
        tau_trace=trace[: 2 * it].reshape(-1, 2), learned_trainings=out.learned_trainings,
        learned_uses=out.learned_uses, learned_r2=out.learned_r2,
        learned_seconds=out.learned_seconds)


@dataclass
class LocoChromResult:
    """LocoChromResult (loco.rs:25-39)."""
    chrom: str
    tau: np.ndarray
    mu: np.ndarray
    residuals: np.ndarray
    working_weights: np.ndarray
    alpha: np.ndarray
    iterations: int = 0
    converged: bool = False
    n_kv: int = 0
    seconds: float = 0.0


def run_loco(y, x, grm: OnTheFlyGrm, marker_chroms: Sequence[str], trait_type: TraitType,
             config: AiRemlConfig = AiRemlConfig()) -> dict:
    """run_loco (loco.rs:54-117) over the GRM handle's markers: marker_chroms gives the
    chromosome of each GRM marker; one fit per chromosome (sorted by name, as the
    reference sorts them) with that chromosome left out of the GRM.  Returns
    {chrom: LocoChromResult}."""
    yy = _f64(y)
    n = yy.size
    if n != grm.n_samples:
        raise SaigeError(_lib.EINVAL, "y.len() != n_samples")
    names = [str(c) for c in marker_chroms]
    if len(names) != grm.n_markers:
        raise SaigeError(_lib.EINVAL, "one chromosome per GRM marker is required")
    chroms = sorted(set(names))
    code = {c: k for k, c in enumerate(chroms)}
    mc = np.array([code[c] for c in names], dtype=np.int32)
    xc, p = _design(x, n)
    cfg = _lib.AiRemlConfigC(config.max_iter, config.tol, config.pcg_tol, config.pcg_max_iter,
                             config.n_random_vectors, config.seed, config.precision, config.solve,
                             config.warm_start, config.precond)
    k = len(chroms)
    outs = (_lib.AiRemlSummaryC * k)()
    alpha = np.zeros((k, p))
    mu = np.zeros((k, n))
    w = np.zeros((k, n))
    check(LIB.saige_fit_loco(grm._h, mc.ctypes.data_as(C.POINTER(C.c_int32)), k, _dptr(yy),
                             _dptr(xc), n, p, int(trait_type), C.byref(cfg), outs, _dptr(alpha),
                             _dptr(mu), _dptr(w)))
    res = {}
    for i, c in enumerate(chroms):
        o = outs[i]
        res[c] = LocoChromResult(c, np.array([o.tau[0], o.tau[1]]), mu[i].copy(), yy - mu[i],
                                 w[i].copy(), alpha[i].copy(), o.iterations, bool(o.converged),
                                 o.n_kv, o.seconds)
    return res


# ---------------------------------------------------------------------------
# synthetic cohorts
# ---------------------------------------------------------------------------
@dataclass
class CohortSpec:
    seed: int = 12345
    n: int = 2000
    m: int = 5000
    sib_frac: float = 0.10
    cousin_frac: float = 0.0
    missing_rate: float = 0.01
    maf_lo: float = 0.01
    maf_hi: float = 0.5
    trait: int = _lib.TRAIT_BINARY
    n_covar: int = 2
    prevalence: float = 0.10
    h2: float = 0.2
    n_causal: int = 500

    def c(self) -> _lib.CohortSpecC:
        return _lib.CohortSpecC(self.seed, self.n, self.m, self.sib_frac, self.cousin_frac,
                                self.missing_rate, self.maf_lo, self.maf_hi, self.trait,
                                self.n_covar, self.prevalence, self.h2, self.n_causal, 0)

    @property
    def bed_len(self) -> int:
        return 3 + self.m * ((self.n + 3) // 4)


def gen_bed(spec: CohortSpec) -> np.ndarray:
    out = np.empty(spec.bed_len, dtype=np.uint8)
    s = spec.c()
    check(LIB.saige_gen_bed(C.byref(s), out.ctypes.data_as(C.c_void_p), 0))
    return out


def gen_bed_dev(spec: CohortSpec, dev_ptr: int) -> None:
    s = spec.c()
    check(LIB.saige_gen_bed(C.byref(s), C.c_void_p(dev_ptr), 1))


def gen_pheno(spec: CohortSpec) -> tuple[np.ndarray, np.ndarray]:
    """(y, x) with x n x (1 + n_covar), intercept first, column-major (the layout of
    saige-rs's nalgebra matrices and of this library's C ABI)."""
    y = np.empty(spec.n)
    x = np.empty(spec.n * (1 + spec.n_covar))
    s = spec.c()
    check(LIB.saige_gen_pheno(C.byref(s), _dptr(y), _dptr(x)))
    return y, x.reshape(1 + spec.n_covar, spec.n).T


# ---------------------------------------------------------------------------
# variance ratio (variance_ratio.rs:87-246, fit_null.rs:290-373)
# ---------------------------------------------------------------------------
VR_XADJUST_REFERENCE = 0   # (X'WX)^-1 X'W laid out as fit_null.rs:294-306 builds it
VR_XADJUST_PROJECTION = 1  # the projection X (X'WX)^-1 X'W g


@dataclass
class VarianceRatioConfig:
    """VarianceRatioConfig (variance_ratio.rs:28-56) plus the solver settings."""
    n_markers: int = 30
    min_mac: float = 20.0
    use_categorical: bool = False
    ratio_cv_cutoff: float = 0.001
    seed: int = 12345
    precision: int = PREC_FP32
    xadjust: int = VR_XADJUST_REFERENCE
    block: int = 0  # candidates per block PCG; 0: 64 for MIXED, else n_markers then 10

    def c(self) -> "_lib.VrConfigC":
        return _lib.VrConfigC(self.n_markers, int(self.use_categorical), self.min_mac,
                              self.ratio_cv_cutoff, self.seed, self.precision, self.xadjust,
                              self.block, 0)


@dataclass
class VarianceRatioResult:
    """VarianceRatioResult (variance_ratio.rs:59-71) plus work counters."""
    variance_ratio: float
    categorical_vr: list
    n_markers_used: int
    per_marker_vr: np.ndarray
    used_idx: np.ndarray
    n_solved: int = 0
    n_blocks: int = 0
    pcg_iters: int = 0
    n_kv: int = 0
    seconds: float = 0.0


def vr_marker_order(seed: int, n_cand: int) -> np.ndarray:
    """Order in which estimate_variance_ratio tries its candidates (variance_ratio.rs:116-120)."""
    out = np.empty(max(n_cand, 0), dtype=np.int64)
    check(LIB.saige_vr_marker_order(seed, n_cand, _i64ptr(out)))
    return out


def estimate_variance_ratio(grm: "OnTheFlyGrm", dosage_vectors, mac_values, mu, working_weights,
                            tau, trait_type: TraitType, x,
                            config: VarianceRatioConfig = VarianceRatioConfig()
                            ) -> VarianceRatioResult:
    """estimate_variance_ratio with Sigma^-1 = (tau0 diag(1/w) + tau1 K)^-1 over the GRM
    handle and XVX_inv_XV built from the working weights, as fit_null.rs:290-342 does.
    dosage_vectors: (n_cand, n) with NaN for missing calls; x: (n, p)."""
    d = np.ascontiguousarray(dosage_vectors, dtype=np.float64)
    if d.ndim == 1:
        d = d[None, :]
    n_cand = d.shape[0] if d.size else 0
    mac = _f64(mac_values, n_cand)
    n = grm.n_samples
    mu_ = _f64(mu, n)
    w_ = _f64(working_weights, n)
    t = _f64(tau, 2)
    xa = np.asarray(x, dtype=np.float64)
    if xa.ndim == 1:
        xa = xa[:, None]
    p = xa.shape[1]
    xc = np.ascontiguousarray(xa.T)  # column-major n x p
    cfg = config.c()
    out = _lib.VrSummaryC()
    vr = np.empty(max(n_cand, 1))
    used = np.empty(max(n_cand, 1), dtype=np.int64)
    check(LIB.saige_estimate_variance_ratio(grm._h, _dptr(d), _dptr(mac), n_cand, _dptr(mu_),
                                            _dptr(w_), _dptr(t), int(trait_type), _dptr(xc), p,
                                            C.byref(cfg), C.byref(out), _dptr(vr),
                                            _i64ptr(used)))
    k = out.n_markers_used
    cats = [(out.cat_upper[i], out.cat_vr[i]) for i in range(out.n_categories)]
    return VarianceRatioResult(out.variance_ratio, cats, k, vr[:k].copy(), used[:k].copy(),
                               out.n_solved, out.n_blocks, out.pcg_iters, out.n_kv, out.seconds)


def write_variance_ratio_file(result: VarianceRatioResult, path) -> None:
    """write_variance_ratio_file (variance_ratio.rs:322-338): "<vr> null 1", or one line
    per MAC category "<vr> null <k>"."""
    with open(path, "w") as f:
        if not result.categorical_vr:
            f.write(f"{_rust_f64(result.variance_ratio)} null 1\n")
        else:
            for k, (_, vr) in enumerate(result.categorical_vr):
                f.write(f"{_rust_f64(vr)} null {k + 1}\n")


def _rust_f64(x: float) -> str:
    """Rust's Display for f64: the shortest repr that round-trips, no exponent for
    ordinary magnitudes, integers without a fractional part (1.0 -> "1")."""
    if x != x:
        return "NaN"
    if x in (float("inf"), float("-inf")):
        return "inf" if x > 0 else "-inf"
    if x == int(x) and abs(x) < 1e16:
        return str(int(x))
    r = repr(x)
    if "e" in r:
        mant, exp = r.split("e")
        e = int(exp)
        digits = mant.replace("-", "").replace(".", "")
        sign = "-" if x < 0 else ""
        point = mant.replace("-", "").find(".")
        point = len(mant.replace("-", "")) if point < 0 else point
        pos = point + e
        if pos <= 0:
            return sign + "0." + "0" * (-pos) + digits
        if pos >= len(digits):
            return sign + digits + "0" * (pos - len(digits))
        return sign + digits[:pos] + "." + digits[pos:]
    return r


# ---------------------------------------------------------------------------
# the .saige.model file (null_model.rs:17-113, serialization.rs:13-34)
# ---------------------------------------------------------------------------
@dataclass
class NullModel:
    """NullModel (null_model.rs:17-60)."""
    trait_type: TraitType
    sample_ids: list
    tau: np.ndarray
    alpha: np.ndarray
    mu: np.ndarray
    mu2: np.ndarray
    residuals: np.ndarray
    y: np.ndarray
    x_flat: np.ndarray
    x_ncols: int
    xvx_inv_xv_flat: np.ndarray
    variance_ratio: VarianceRatioResult
    magic: bytes = b"SGMD"
    version: int = 1
    n_samples: int = 0
    n_covariates: int = 0
    use_loco: bool = False
    loco_tau: list = field(default_factory=list)
    loco_mu: list = field(default_factory=list)
    loco_residuals: list = field(default_factory=list)
    use_sparse_grm: bool = False
    n_markers_in_grm: int = 0


def xvx_inv_xv(x, working_weights) -> np.ndarray:
    """(X'WX)^-1 X'W laid out as fit_null.rs:290-305 fills it: a flat p*n array with
    element (j, i) at j*n + i.  x is n x p."""
    xa = np.asarray(x, dtype=np.float64)
    if xa.ndim == 1:
        xa = xa[:, None]
    n, p = xa.shape
    xc = np.ascontiguousarray(xa.T)
    out = np.empty(p * n)
    check(LIB.saige_xvx_inv_xv(_dptr(xc), _dptr(_f64(working_weights, n)), n, p, _dptr(out)))
    return out


def save_model(path, trait_type: TraitType, sample_ids: Sequence[str], tau, alpha, mu, y, x,
               xvx_inv_xv_flat, vr: VarianceRatioResult, loco: Optional[dict] = None,
               n_markers_in_grm: int = 0, use_sparse_grm: bool = False) -> None:
    """save_model(NullModel::new(...)) (serialization.rs:13-17, null_model.rs:71-112):
    the bincode file saige-rs Step 2 loads.  loco: {chrom: LocoChromResult} (fit_null
    itself writes none)."""
    yy = _f64(y)
    n = yy.size
    xa = np.asarray(x, dtype=np.float64)
    if xa.ndim == 1:
        xa = xa[:, None]
    p = xa.shape[1]
    keep = []  # owners of the buffers the struct points to

    def dp(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return _dptr(a)

    def sp(strs):
        arr = (C.c_char_p * max(len(strs), 1))(*[str(t).encode() for t in strs])
        keep.append(arr)
        return C.cast(arr, C.POINTER(C.c_char_p))

    m = _lib.NullModelC()
    m.trait = int(trait_type)
    m.p = p
    m.n = n
    m.sample_ids = sp(list(sample_ids))
    if len(sample_ids) != n:
        raise SaigeError(_lib.EINVAL, "one sample id per sample is required")
    m.tau[0], m.tau[1] = float(tau[0]), float(tau[1])
    m.alpha = dp(_f64(alpha, p))
    m.mu = dp(_f64(mu, n))
    m.y = dp(yy)
    m.x = dp(np.ascontiguousarray(xa.T).ravel())
    m.xvx_inv_xv = dp(_f64(xvx_inv_xv_flat, p * n))
    m.variance_ratio = vr.variance_ratio
    m.vr_n_categories = len(vr.categorical_vr)
    m.vr_cat_upper = dp(np.array([c[0] for c in vr.categorical_vr] or [0.0]))
    m.vr_cat_vr = dp(np.array([c[1] for c in vr.categorical_vr] or [0.0]))
    m.vr_n_markers_used = vr.n_markers_used
    per = np.asarray(vr.per_marker_vr, dtype=np.float64)
    m.vr_per_marker = dp(per if per.size else np.zeros(1))
    m.vr_n_per_marker = per.size
    loco = loco or {}
    chroms = list(loco.keys())
    m.use_loco = 1 if chroms else 0
    m.n_loco = len(chroms)
    m.loco_chrom = sp(chroms)
    m.loco_tau = dp(np.array([loco[c].tau for c in chroms]).ravel() if chroms else np.zeros(1))
    m.loco_mu = dp(np.array([loco[c].mu for c in chroms]).ravel() if chroms else np.zeros(1))
    m.loco_residuals = dp(np.array([loco[c].residuals for c in chroms]).ravel()
                          if chroms else np.zeros(1))
    m.use_sparse_grm = int(use_sparse_grm)
    m.n_markers_in_grm = n_markers_in_grm
    check(LIB.saige_write_null_model(str(path).encode(), C.byref(m)))


class _Reader:
    def __init__(self, data: bytes):
        self.d, self.o = memoryview(data), 0

    def take(self, k):
        if self.o + k > len(self.d):
            raise ValueError("truncated model file")
        b = self.d[self.o:self.o + k]
        self.o += k
        return b

    def u8(self):
        return self.take(1)[0]

    def u32(self):
        return int.from_bytes(self.take(4), "little")

    def u64(self):
        return int.from_bytes(self.take(8), "little")

    def f64(self):
        return float(np.frombuffer(self.take(8), dtype="<f8")[0])

    def vec(self):
        k = self.u64()
        return np.frombuffer(self.take(8 * k), dtype="<f8").copy()

    def str(self):
        return bytes(self.take(self.u64())).decode()


def load_model(path) -> NullModel:
    """load_model (serialization.rs:20-34): bincode decode, then the magic check."""
    r = _Reader(open(path, "rb").read())
    magic = bytes(r.take(4))
    version = r.u32()
    trait = TraitType(r.u32())
    ids = [r.str() for _ in range(r.u64())]
    n_samples, n_cov = r.u64(), r.u64()
    tau = np.array([r.f64(), r.f64()])
    alpha, mu, mu2, resid, y, x = r.vec(), r.vec(), r.vec(), r.vec(), r.vec(), r.vec()
    x_ncols = r.u64()
    xvx = r.vec()
    vr_val = r.f64()
    cats = [(r.f64(), r.f64()) for _ in range(r.u64())]
    n_used = r.u64()
    per = r.vec()
    use_loco = bool(r.u8())
    loco_tau = [(r.str(), (r.f64(), r.f64())) for _ in range(r.u64())]
    loco_mu = [(r.str(), r.vec()) for _ in range(r.u64())]
    loco_res = [(r.str(), r.vec()) for _ in range(r.u64())]
    sparse = bool(r.u8())
    n_grm = r.u64()
    if magic != b"SGMD":
        raise ValueError(f"Invalid model file: expected magic bytes b'SGMD', got {magic!r}")
    vr = VarianceRatioResult(vr_val, cats, n_used, per, np.zeros(0, np.int64))
    return NullModel(trait, ids, tau, alpha, mu, mu2, resid, y, x, x_ncols, xvx, vr, magic,
                     version, n_samples, n_cov, use_loco, loco_tau, loco_mu, loco_res, sparse,
                     n_grm)


# ---------------------------------------------------------------------------
# whole fit-null from host buffers, instrumentation
# ---------------------------------------------------------------------------
@dataclass
class FitNullResult:
    ai_reml: AiRemlResult
    m_grm: int
    m_vr: int
    variance_ratio: Optional["VarianceRatioResult"] = None


def fit_null_from_bed(bed, n_fam: int, m_tot: int, y, x, trait_type: TraitType,
                      config: AiRemlConfig = AiRemlConfig(), sample_idx=None,
                      min_maf: float = 0.01, max_missing: float = 0.15,
                      variance_ratio: bool = False,
                      vr_config: Optional[VarianceRatioConfig] = None) -> FitNullResult:
    """Marker statistics, QC + VR/GRM split, GRM operator and AI-REML in one call
    (the genotype part of saige-cli fit_null::run), followed by the variance ratio
    over the VR candidates when variance_ratio is true (fit_null.rs:290-373)."""
    b = _bed_array(bed)
    yy = _f64(y)
    n = yy.size
    xc, p = _design(x, n)
    sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
    cfg = _lib.AiRemlConfigC(config.max_iter, config.tol, config.pcg_tol, config.pcg_max_iter,
                             config.n_random_vectors, config.seed, config.precision, config.solve,
                             config.warm_start, config.precond)
    out = _lib.AiRemlSummaryC()
    alpha = np.zeros(p)
    mu = np.zeros(n)
    trace = np.full(2 * max(config.max_iter, 1), np.nan)
    mg, mv = C.c_int64(), C.c_int64()
    vsum = _lib.VrSummaryC()
    vcfg = None
    if vr_config is not None:
        vcfg = vr_config.c()
    check(LIB.saige_fit_null_from_bed(
        b.ctypes.data_as(C.POINTER(C.c_uint8)), b.size, n_fam, m_tot, _i64ptr(sidx), n, _dptr(yy),
        _dptr(xc), p, int(trait_type), min_maf, max_missing, C.byref(cfg), C.byref(out),
        _dptr(alpha), _dptr(mu), _dptr(trace), C.byref(mg), C.byref(mv),
        C.byref(vcfg) if vcfg is not None else None,
        C.byref(vsum) if variance_ratio else None))
    it = out.iterations
    res = AiRemlResult(
        tau=np.array([out.tau[0], out.tau[1]]), iterations=it, converged=bool(out.converged),
        mu=mu, working_weights=np.zeros(0), residuals=yy - mu, eta=np.zeros(0), alpha=alpha,
        log_likelihood=out.log_likelihood, n_kv=out.n_kv, n_kv_launches=out.n_kv_launches,
        pcg_iters=out.pcg_iters, seconds=out.seconds, tau_trace=trace[: 2 * it].reshape(-1, 2))
    vr = None
    if variance_ratio:
        cats = [(vsum.cat_upper[i], vsum.cat_vr[i]) for i in range(vsum.n_categories)]
        vr = VarianceRatioResult(vsum.variance_ratio, cats, vsum.n_markers_used, np.zeros(0),
                                 np.zeros(0, np.int64), vsum.n_solved, vsum.n_blocks,
                                 vsum.pcg_iters, vsum.n_kv, vsum.seconds)
    return FitNullResult(res, mg.value, mv.value, vr)


@dataclass
class CohortFit:
    tau: np.ndarray
    iterations: int
    converged: bool
    alpha: np.ndarray
    m_grm: int
    n_kv_launches: int
    pcg_iters: int
    seconds: float


def fit_null_cohorts(bed, n_fam: int, m_tot: int, cohorts, trait_type: TraitType,
                     config: AiRemlConfig = AiRemlConfig(), min_maf: float = 0.01,
                     max_missing: float = 0.15, concurrent: bool = True):
    """fit_null::run (genotype part, no variance ratio) for each sub-cohort of one .bed.
    cohorts: sequence of (sample_idx, y, x).  Returns ([CohortFit], wall seconds); with
    concurrent the cohorts run on their own threads and streams."""
    b = _bed_array(bed)
    k = len(cohorts)
    sidx = [np.ascontiguousarray(c[0], dtype=np.int64) for c in cohorts]
    ys = [_f64(c[1]) for c in cohorts]
    xs, ps = zip(*[_design(c[2], ys[i].size) for i, c in enumerate(cohorts)])
    if len(set(ps)) != 1:
        raise SaigeError(_lib.EINVAL, "every cohort needs the same covariate count")
    p = ps[0]
    alphas = [np.zeros(p) for _ in range(k)]
    P = C.POINTER
    s_arr = (P(C.c_int64) * k)(*[_i64ptr(a) for a in sidx])
    n_arr = np.array([a.size for a in sidx], dtype=np.int64)
    y_arr = (P(C.c_double) * k)(*[_dptr(a) for a in ys])
    x_arr = (P(C.c_double) * k)(*[_dptr(a) for a in xs])
    a_arr = (P(C.c_double) * k)(*[_dptr(a) for a in alphas])
    outs = (_lib.AiRemlSummaryC * k)()
    mg = np.zeros(k, dtype=np.int64)
    wall = C.c_double(0.0)
    cfg = _lib.AiRemlConfigC(config.max_iter, config.tol, config.pcg_tol, config.pcg_max_iter,
                             config.n_random_vectors, config.seed, config.precision, config.solve,
                             config.warm_start, config.precond)
    check(LIB.saige_fit_null_cohorts(
        b.ctypes.data_as(C.POINTER(C.c_uint8)), b.size, n_fam, m_tot, k, s_arr, _i64ptr(n_arr),
        y_arr, x_arr, p, int(trait_type), min_maf, max_missing, C.byref(cfg), 1 if concurrent else 0,
        outs, a_arr, _i64ptr(mg), C.byref(wall)))
    res = [CohortFit(np.array([o.tau[0], o.tau[1]]), o.iterations, bool(o.converged), alphas[i],
                     int(mg[i]), o.n_kv_launches, o.pcg_iters, o.seconds)
           for i, o in enumerate(outs)]
    return res, wall.value


def _with_extension(prefix, ext: str) -> str:
    """std::path::Path::with_extension: replace (or add) the last component's extension."""
    import os
    head, tail = os.path.split(str(prefix))
    dot = tail.rfind(".")
    stem = tail[:dot] if dot > 0 else tail
    return os.path.join(head, f"{stem}.{ext}")


def save_fit_null(prefix, result: FitNullResult, trait_type: TraitType, sample_ids, y, x) -> tuple:
    """The files fit_null::run writes (fit_null.rs:376-399): <prefix>.varianceRatio.txt and
    <prefix>.saige.model, from a fit_null_from_bed result with its variance ratio.  The
    working weights are max(V(mu), 1e-30) (family.rs:55-66)."""
    if result.variance_ratio is None:
        raise SaigeError(_lib.EINVAL, "the result holds no variance ratio")
    mu = result.ai_reml.mu
    w = np.maximum(mu * (1 - mu) if trait_type != TraitType.Quantitative
                   else np.ones_like(mu), 1e-30)
    vr_path = _with_extension(prefix, "varianceRatio.txt")
    model_path = _with_extension(prefix, "saige.model")
    write_variance_ratio_file(result.variance_ratio, vr_path)
    save_model(model_path, trait_type, sample_ids, result.ai_reml.tau, result.ai_reml.alpha, mu,
               y, x, xvx_inv_xv(x, w), result.variance_ratio)
    return model_path, vr_path


def kernel_launches() -> int:
    return int(LIB.saige_kernel_launches())


def _grm_stats(self) -> dict:
    st = _lib.GrmStatsC()
    check(LIB.saige_grm_get_stats(self._h, C.byref(st)))
    return {f: getattr(st, f) for f, _ in _lib.GrmStatsC._fields_}


def _grm_set_profiling(self, on: bool = True) -> None:
    check(LIB.saige_grm_set_profiling(self._h, 1 if on else 0))


def _grm_reset_stats(self) -> None:
    check(LIB.saige_grm_reset_stats(self._h))


OnTheFlyGrm.stats = _grm_stats
OnTheFlyGrm.set_profiling = _grm_set_profiling
OnTheFlyGrm.reset_stats = _grm_reset_stats
