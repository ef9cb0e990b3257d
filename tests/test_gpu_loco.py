"""Leave-one-chromosome-out fits (loco.rs:54-117) on the GPU, through the C ABI.

The LOCO fits share the handle's packed genotypes and leave the chromosome's
markers out of every product.  In MIXED precision the products are exact integer
sums plus the same FP64 epilogue, so each LOCO fit must equal, bit for bit, the fit
on a GRM built from the remaining markers; FP32 products sum in another order, so
they are held to the FP32 tolerance; the FP64 oracle pins tau."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cohort():
    n, m = 1000, 900
    spec = cs.CohortSpec(n=n, m=m, seed=23, prevalence=0.25, h2=0.4, n_covar=2)
    bed = cs.gen_bed(spec)
    af, mac, nv = O.marker_stats(bed, n, m)
    keep = np.nonzero((af >= 0.01) & (af <= 0.99))[0]
    # three chromosomes named so that string order differs from numeric order
    names = np.where(keep < 300, "1", np.where(keep < 600, "2", "10"))
    y, x = cs.gen_pheno(spec)
    return dict(bed=bed, n=n, m=m, af=af, keep=keep, names=names, y=y, x=x)


def _grm(c, idx, precision):
    return cs.OnTheFlyGrm.from_bed(c["bed"], c["n"], c["m"], idx, c["af"][idx],
                                   precision=precision)


def test_loco_chromosomes_in_reference_order(cohort):
    c = cohort
    grm = _grm(c, c["keep"], cs.PREC_MIXED)
    cfg = cs.AiRemlConfig(max_iter=2, precision=cs.PREC_MIXED)
    res = cs.run_loco(c["y"], c["x"], grm, list(c["names"]), cs.TraitType.Binary, cfg)
    assert list(res.keys()) == ["1", "10", "2"]


@pytest.mark.parametrize("solve,warm", [(cs.SOLVE_SINGLE, cs.WARM_ZERO),
                                        (cs.SOLVE_BLOCK, cs.WARM_PREVIOUS),
                                        (cs.SOLVE_BLOCK, cs.WARM_RECYCLED)])
def test_mixed_loco_equals_refit_without_the_chromosome(cohort, solve, warm):
    c = cohort
    cfg = cs.AiRemlConfig(max_iter=4, precision=cs.PREC_MIXED, solve=solve, warm_start=warm)
    grm = _grm(c, c["keep"], cs.PREC_MIXED)
    res = cs.run_loco(c["y"], c["x"], grm, list(c["names"]), cs.TraitType.Binary, cfg)
    for chrom, r in res.items():
        rest = c["keep"][c["names"] != chrom]
        ref = cs.fit_ai_reml(c["y"], c["x"], _grm(c, rest, cs.PREC_MIXED),
                             cs.TraitType.Binary, cfg)
        assert np.array_equal(r.tau, ref.tau), chrom
        assert np.array_equal(r.mu, ref.mu), chrom
        assert np.array_equal(r.alpha, ref.alpha), chrom


def test_fp32_loco_matches_refit_and_oracle(cohort):
    c = cohort
    cfg = cs.AiRemlConfig(max_iter=6, tol=1e-5)
    grm = _grm(c, c["keep"], cs.PREC_FP32)
    res = cs.run_loco(c["y"], c["x"], grm, list(c["names"]), cs.TraitType.Binary, cfg)
    chrom = "2"
    rest = c["keep"][c["names"] != chrom]
    ref = cs.fit_ai_reml(c["y"], c["x"], _grm(c, rest, cs.PREC_FP32), cs.TraitType.Binary, cfg)
    assert abs(res[chrom].tau[1] - ref.tau[1]) <= 1e-5 * abs(ref.tau[1])
    z = O.standardize(O.dosages(c["bed"], c["n"], rest), c["af"][rest], 0)
    orc = O.fit_ai_reml(c["y"], c["x"], O.BINARY, O.K_EXPLICIT, O.grm_explicit(z), max_iter=6,
                        tol=1e-5)
    assert abs(res[chrom].tau[1] - orc["tau"][1]) <= 1e-4 * abs(orc["tau"][1])
