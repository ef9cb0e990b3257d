"""ctypes binding of libsaige_gpu.so (include/saige_gpu.h).

The shared library is the product: there is no Python or CPU fallback.  If it
is missing, importing this module raises with the command that builds it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libsaige_gpu.so"

OK, EINVAL, ENOMEM, ECUDA, NOT_CONVERGED, TIMEOUT, SINGULAR, EBED, ENOTSUP = range(9)
STATUS_NAMES = {
    0: "SAIGE_OK",
    1: "SAIGE_EINVAL",
    2: "SAIGE_ENOMEM",
    3: "SAIGE_ECUDA",
    4: "SAIGE_NOT_CONVERGED",
    5: "SAIGE_TIMEOUT",
    6: "SAIGE_SINGULAR",
    7: "SAIGE_EBED",
    8: "SAIGE_ENOTSUP",
}

PREC_FP32, PREC_MIXED = 0, 1
TRAIT_BINARY, TRAIT_QUANTITATIVE, TRAIT_SURVIVAL = 0, 1, 2
SOLVE_SINGLE, SOLVE_BLOCK = 0, 1
WARM_ZERO, WARM_PREVIOUS, WARM_LEARNED, WARM_RECYCLED = 0, 1, 2, 3


class SaigeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class PcgOptions(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_iter", C.c_int32), ("precision", C.c_int32)]


class AiRemlConfigC(C.Structure):
    _fields_ = [
        ("max_iter", C.c_int32),
        ("tol", C.c_double),
        ("pcg_tol", C.c_double),
        ("pcg_max_iter", C.c_int32),
        ("n_random_vectors", C.c_int32),
        ("seed", C.c_uint64),
        ("precision", C.c_int32),
        ("solve", C.c_int32),
        ("warm_start", C.c_int32),
        ("precond", C.c_int32),
    ]


class AiRemlSummaryC(C.Structure):
    _fields_ = [
        ("tau", C.c_double * 2),
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("log_likelihood", C.c_double),
        ("n_kv", C.c_int64),
        ("n_kv_launches", C.c_int64),
        ("pcg_iters", C.c_int64),
        ("seconds", C.c_double),
        ("learned_trainings", C.c_int32),
        ("learned_uses", C.c_int32),
        ("learned_r2", C.c_double),
        ("learned_seconds", C.c_double),
    ]


class ExplicitGrmConfigC(C.Structure):
    _fields_ = [
        ("min_maf", C.c_double),
        ("relatedness_cutoff", C.c_double),
        ("arith", C.c_int32),
        ("device", C.c_int32),
        ("reserved", C.c_int32 * 4),
    ]


class ExplicitGrmInfoC(C.Structure):
    _fields_ = [
        ("n_markers_used", C.c_int64),
        ("nnz", C.c_int64),
        ("kernel_seconds", C.c_double),
        ("total_seconds", C.c_double),
        ("terms", C.c_double),
    ]


class VrConfigC(C.Structure):
    _fields_ = [
        ("n_markers", C.c_int32),
        ("use_categorical", C.c_int32),
        ("min_mac", C.c_double),
        ("ratio_cv_cutoff", C.c_double),
        ("seed", C.c_uint64),
        ("precision", C.c_int32),
        ("xadjust", C.c_int32),
        ("block", C.c_int32),
        ("reserved", C.c_int32),
    ]


class VrSummaryC(C.Structure):
    _fields_ = [
        ("variance_ratio", C.c_double),
        ("n_markers_used", C.c_int32),
        ("n_categories", C.c_int32),
        ("cat_upper", C.c_double * 8),
        ("cat_vr", C.c_double * 8),
        ("n_solved", C.c_int32),
        ("n_blocks", C.c_int32),
        ("pcg_iters", C.c_int64),
        ("n_kv", C.c_int64),
        ("seconds", C.c_double),
    ]


class NullModelC(C.Structure):
    _fields_ = [
        ("trait", C.c_int32),
        ("p", C.c_int32),
        ("n", C.c_int64),
        ("sample_ids", C.POINTER(C.c_char_p)),
        ("tau", C.c_double * 2),
        ("alpha", C.POINTER(C.c_double)),
        ("mu", C.POINTER(C.c_double)),
        ("y", C.POINTER(C.c_double)),
        ("x", C.POINTER(C.c_double)),
        ("xvx_inv_xv", C.POINTER(C.c_double)),
        ("variance_ratio", C.c_double),
        ("vr_n_categories", C.c_int32),
        ("use_loco", C.c_int32),
        ("vr_cat_upper", C.POINTER(C.c_double)),
        ("vr_cat_vr", C.POINTER(C.c_double)),
        ("vr_n_markers_used", C.c_int64),
        ("vr_per_marker", C.POINTER(C.c_double)),
        ("vr_n_per_marker", C.c_int64),
        ("n_loco", C.c_int32),
        ("use_sparse_grm", C.c_int32),
        ("loco_chrom", C.POINTER(C.c_char_p)),
        ("loco_tau", C.POINTER(C.c_double)),
        ("loco_mu", C.POINTER(C.c_double)),
        ("loco_residuals", C.POINTER(C.c_double)),
        ("n_markers_in_grm", C.c_int64),
    ]


class GrmStatsC(C.Structure):
    _fields_ = [
        ("n_kv", C.c_int64),
        ("n_kv_launches", C.c_int64),
        ("tc_pass_a_launches", C.c_int64),
        ("tc_pass_b_launches", C.c_int64),
        ("tc_pass_a_ms", C.c_double),
        ("tc_pass_b_ms", C.c_double),
        ("fp32_launches", C.c_int64),
        ("fp32_ms", C.c_double),
        ("sc_launches", C.c_int64),
        ("sc_ms", C.c_double),
        ("sc_list_launches", C.c_int64),
        ("missing_listed", C.c_int64),
    ]


class CohortSpecC(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("n", C.c_int64),
        ("m", C.c_int64),
        ("sib_frac", C.c_double),
        ("cousin_frac", C.c_double),
        ("missing_rate", C.c_double),
        ("maf_lo", C.c_double),
        ("maf_hi", C.c_double),
        ("trait", C.c_int32),
        ("n_covar", C.c_int32),
        ("prevalence", C.c_double),
        ("h2", C.c_double),
        ("n_causal", C.c_int32),
        ("reserved", C.c_int32),
    ]


P = C.POINTER
_d, _i64, _i32, _u8, _u64, _sz, _vp = (
    P(C.c_double),
    P(C.c_int64),
    P(C.c_int32),
    P(C.c_uint8),
    C.c_uint64,
    C.c_size_t,
    C.c_void_p,
)

# name -> (restype, argtypes), exactly the declarations of include/saige_gpu.h
SIGNATURES = {
    "saige_last_error": (C.c_char_p, []),
    "saige_version": (C.c_int32, []),
    "saige_device_count": (C.c_int32, []),
    "saige_bed_marker_stats": (
        C.c_int32,
        [_u8, _sz, C.c_int64, C.c_int64, _i64, C.c_int64, _d, _d, _i64],
    ),
    "saige_select_grm_markers": (
        C.c_int32,
        [_d, _d, _i64, C.c_int64, C.c_int64, C.c_double, C.c_double, _u64, _i64, _i64, _i64, _i64],
    ),
    "saige_grm_create_from_bed": (
        C.c_int32,
        [_u8, _sz, C.c_int64, C.c_int64, _i64, C.c_int64, _i64, C.c_int64, _d, C.c_int32, P(_vp)],
    ),
    "saige_grm_create_from_bed_dev": (
        C.c_int32,
        [_vp, _sz, C.c_int64, C.c_int64, _i64, C.c_int64, _i64, C.c_int64, _d, C.c_int32, P(_vp)],
    ),
    "saige_grm_create_from_dosages": (
        C.c_int32,
        [_d, C.c_int64, C.c_int64, _d, C.c_int32, P(_vp)],
    ),
    "saige_grm_destroy": (C.c_int32, [_vp]),
    "saige_grm_dims": (C.c_int32, [_vp, _i64, _i64]),
    "saige_grm_matvec": (C.c_int32, [_vp, _d, _d, C.c_int64, C.c_int32, C.c_int32]),
    "saige_grm_matvec_dev": (
        C.c_int32,
        [_vp, _vp, _vp, C.c_int64, C.c_int32, C.c_int32, _vp],
    ),
    "saige_grm_diag": (C.c_int32, [_vp, _d, C.c_int64]),
    "saige_tc_set_wait_budget": (C.c_int32, [C.c_int64]),
    "saige_grm_noalloc_scratch_bytes": (C.c_int32, [_vp, P(_sz), P(_sz)]),
    "saige_release_cached_memory": (C.c_int32, []),
    "saige_write_null_model": (C.c_int32, [C.c_char_p, P(NullModelC)]),
    "saige_xvx_inv_xv": (C.c_int32, [_d, _d, C.c_int64, C.c_int32, _d]),
    "saige_fit_null_cohorts": (
        C.c_int32,
        [_u8, _sz, C.c_int64, C.c_int64, C.c_int32, P(_i64), _i64, P(_d), P(_d), C.c_int32,
         C.c_int32, C.c_double, C.c_double, P(AiRemlConfigC), C.c_int32, P(AiRemlSummaryC), P(_d),
         _i64, _d],
    ),
    "saige_mlp_param_count": (C.c_int32, []),
    "saige_mlp_initial_params": (C.c_int32, [C.c_uint64, P(C.c_float)]),
    "saige_mlp_eval": (C.c_int32, [P(C.c_float), P(C.c_float), P(C.c_float), C.c_int64,
                                   P(C.c_float), P(C.c_float), _d, C.c_int32]),
    "saige_mlp_train": (C.c_int32, [P(C.c_float), P(C.c_float), P(C.c_float), C.c_int64,
                                    C.c_int32, C.c_int32, C.c_float, C.c_int32, _d, _d, _d,
                                    C.c_int32]),
    "saige_explicit_grm_config_default": (C.c_int32, [P(ExplicitGrmConfigC)]),
    "saige_dense_grm_from_bed": (
        C.c_int32,
        [_u8, C.c_size_t, C.c_int64, C.c_int64, _i64, C.c_int64, P(ExplicitGrmConfigC), _d,
         P(ExplicitGrmInfoC)],
    ),
    "saige_sparse_grm_from_bed": (
        C.c_int32,
        [_u8, C.c_size_t, C.c_int64, C.c_int64, _i64, C.c_int64, P(ExplicitGrmConfigC),
         P(_vp), P(ExplicitGrmInfoC)],
    ),
    "saige_grm_from_dosages": (
        C.c_int32,
        [_d, _d, C.c_int64, C.c_int64, P(ExplicitGrmConfigC), _d, P(ExplicitGrmInfoC)],
    ),
    "saige_sparse_grm_from_dosages": (
        C.c_int32,
        [_d, _d, C.c_int64, C.c_int64, P(ExplicitGrmConfigC), P(_vp), P(ExplicitGrmInfoC)],
    ),
    "saige_sparse_grm_n": (C.c_int64, [_vp]),
    "saige_sparse_grm_nnz": (C.c_int64, [_vp]),
    "saige_sparse_grm_n_markers": (C.c_int64, [_vp]),
    "saige_sparse_grm_get": (C.c_int32, [_vp, P(C.c_int32), P(C.c_int32), _d]),
    "saige_sparse_grm_free": (None, [_vp]),
    "saige_sparse_grm_from_triplets": (
        C.c_int32,
        [C.c_int64, C.c_int64, P(C.c_int32), P(C.c_int32), _d, C.c_int64, P(_vp)],
    ),
    "saige_write_sparse_grm": (
        C.c_int32, [_vp, P(C.c_char_p), C.c_int64, C.c_char_p, C.c_char_p]),
    "saige_vr_config_default": (C.c_int32, [P(VrConfigC)]),
    "saige_vr_marker_order": (C.c_int32, [C.c_uint64, C.c_int64, _i64]),
    "saige_estimate_variance_ratio": (
        C.c_int32,
        [_vp, _d, _d, C.c_int64, _d, _d, _d, C.c_int32, _d, C.c_int32, P(VrConfigC),
         P(VrSummaryC), _d, _i64],
    ),
    "saige_rademacher_probes": (C.c_int32, [C.c_uint64, C.c_int32, C.c_int64, _d, C.c_int32]),
    "saige_grm_matvec_dev_noalloc": (
        C.c_int32,
        [_vp, _vp, _vp, C.c_int64, C.c_int32, _vp],
    ),
    "saige_pcg_solve": (
        C.c_int32,
        [_vp, _d, _d, _d, _d, _d, C.c_int64, C.c_int32, P(PcgOptions), _i32, _d, _u8],
    ),
    "saige_solve_mixed_model_pcg": (
        C.c_int32,
        [_vp, _d, _d, _d, _d, C.c_int64, P(PcgOptions), _i32, _d, _u8],
    ),
    "saige_ai_reml_config_default": (None, [P(AiRemlConfigC)]),
    "saige_fit_ai_reml": (
        C.c_int32,
        [_vp, _d, _d, C.c_int64, C.c_int32, C.c_int32, P(AiRemlConfigC), P(AiRemlSummaryC),
         _d, _d, _d, _d, _d],
    ),
    "saige_bed_marker_stats_dev": (
        C.c_int32,
        [_vp, _sz, C.c_int64, C.c_int64, _i64, C.c_int64, _d, _d, _i64],
    ),
    "saige_fit_loco": (
        C.c_int32,
        [_vp, _i32, C.c_int32, _d, _d, C.c_int64, C.c_int32, C.c_int32, P(AiRemlConfigC),
         P(AiRemlSummaryC), _d, _d, _d],
    ),
    "saige_fit_null_from_bed": (
        C.c_int32,
        [_u8, _sz, C.c_int64, C.c_int64, _i64, C.c_int64, _d, _d, C.c_int32, C.c_int32,
         C.c_double, C.c_double, P(AiRemlConfigC), P(AiRemlSummaryC), _d, _d, _d, _i64, _i64,
         P(VrConfigC), P(VrSummaryC)],
    ),
    "saige_grm_set_profiling": (C.c_int32, [_vp, C.c_int32]),
    "saige_grm_get_stats": (C.c_int32, [_vp, P(GrmStatsC)]),
    "saige_grm_reset_stats": (C.c_int32, [_vp]),
    "saige_kernel_launches": (C.c_int64, []),
    "saige_tc_autotune_trials": (C.c_int64, []),
    "saige_gen_bed": (C.c_int32, [P(CohortSpecC), _vp, C.c_int32]),
    "saige_gen_pheno": (C.c_int32, [P(CohortSpecC), _d, _d]),
}


def load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the sm_100a library first "
            "(python -c 'import __graft_entry__ as g; g.build()')"
        )
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = load()


def check(code: int) -> None:
    if code != OK:
        raise SaigeError(code, LIB.saige_last_error().decode(errors="replace"))
