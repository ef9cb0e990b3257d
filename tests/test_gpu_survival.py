"""The survival trait (TraitType::Survival: cloglog link, saige-core/src/glmm/link.rs:29-100,
family.rs:23-90, tau_e fixed at 1 as for a binary trait, ai_reml.rs:104) on the GPU
against the FP64 oracle.  The outcome is the cohort's 0/1 event indicator."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cohort():
    spec = cs.CohortSpec(n=1500, m=1200, seed=31, prevalence=0.15, h2=0.4, n_covar=2)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = O.marker_stats(bed, spec.n, spec.m)
    g, _ = O.select_markers(af, mac, nv, spec.n)
    k = O.grm_explicit(O.standardize(O.dosages(bed, spec.n, g), af[g], 0))
    o = O.fit_ai_reml(y, x, O.SURVIVAL, O.K_EXPLICIT, k, max_iter=30, tol=1e-5)
    return dict(spec=spec, bed=bed, y=y, x=x, af=af, g=g, o=o)


@pytest.mark.parametrize("precision,solve,warm", [
    (cs.PREC_FP32, cs.SOLVE_SINGLE, cs.WARM_ZERO),
    (cs.PREC_MIXED, cs.SOLVE_SINGLE, cs.WARM_ZERO),
    (cs.PREC_MIXED, cs.SOLVE_BLOCK, cs.WARM_RECYCLED),
])
def test_survival_fit_matches_fp64_oracle(cohort, precision, solve, warm):
    c, o = cohort, cohort["o"]
    s = c["spec"]
    grm = cs.OnTheFlyGrm.from_bed(c["bed"], s.n, s.m, c["g"], c["af"][c["g"]],
                                  precision=precision)
    cfg = cs.AiRemlConfig(max_iter=30, tol=1e-5, precision=precision, solve=solve,
                          warm_start=warm)
    r = cs.fit_ai_reml(c["y"], c["x"], grm, cs.TraitType.Survival, cfg)
    rel = np.abs(r.tau - o["tau"]) / np.abs(o["tau"])
    print("survival tau", r.tau, "oracle", o["tau"], "rel", rel, r.iterations, o["iterations"])
    assert r.converged and o["converged"]
    assert r.tau[0] == 1.0 and o["tau"][1] > 0
    assert np.all(rel <= 1e-4)
    assert np.abs(r.alpha - o["alpha"]).max() <= 1e-4 * np.abs(o["alpha"]).max()
    # the cloglog mean: mu = 1 - exp(-exp(eta)), clamped (link.rs:29-100)
    assert np.abs(r.mu - o["mu"]).max() <= 1e-4
    if warm == cs.WARM_ZERO:
        assert r.iterations == o["iterations"]
