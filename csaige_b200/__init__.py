"""B200 (sm_100a) implementation of the saige-rs fit-null GRM-product path.

The compute lives in libsaige_gpu.so behind a C ABI (include/saige_gpu.h);
this package is its Python mirror of the saige-rs API.
"""
from ._lib import SaigeError, LIB_PATH  # noqa: F401  (raises ImportError when the .so is missing)
from .api import (  # noqa: F401
    PREC_FP32,
    PREC_MIXED,
    SOLVE_BLOCK,
    SOLVE_SINGLE,
    WARM_LEARNED,
    WARM_PREVIOUS,
    WARM_ZERO,
    AiRemlConfig,
    AiRemlResult,
    CohortSpec,
    OnTheFlyGrm,
    PcgResult,
    PcgSolver,
    SaigePcgConfig,
    LocoChromResult,
    TraitType,
    run_loco,
    VarianceRatioConfig,
    VarianceRatioResult,
    estimate_variance_ratio,
    vr_marker_order,
    write_variance_ratio_file,
    bed_marker_stats,
    device_count,
    fit_ai_reml,
    fit_null_from_bed,
    kernel_launches,
    gen_bed,
    gen_bed_dev,
    gen_pheno,
    select_grm_markers,
    solve_mixed_model_pcg,
    version,
)
