"""Warm starts of the AI-REML PCG solves on the GPU (ai_reml.rs:175-306 with the
x0 hook of decomposition.rs:212).

Every start is followed by PCG to the same tolerance (1e-5), so the fit is the same
to that tolerance whatever the start: tau must agree with the zero-start fit and with
the FP64 oracle, and the recycled start (a Galerkin projection onto vectors whose
Sigma-image needs no GRM product) must take fewer product launches than the
previous-iterate start."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu


def _cohort(trait, n=3000, m=2500, seed=7):
    spec = cs.CohortSpec(n=n, m=m, seed=seed, trait=trait, prevalence=0.1, h2=0.4, n_covar=4,
                         sib_frac=0.2, cousin_frac=0.05, missing_rate=0.01)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = cs.bed_marker_stats(bed, n, m)
    g, _ = cs.select_grm_markers(af, mac, nv, n)
    return dict(bed=bed, y=y, x=x, af=af, g=g, n=n, m=m)


def _fit(c, trait, warm, precision=cs.PREC_MIXED, tol=0.02):
    grm = cs.OnTheFlyGrm.from_bed(c["bed"], c["n"], c["m"], c["g"], c["af"][c["g"]],
                                  precision=precision)
    cfg = cs.AiRemlConfig(precision=precision, solve=cs.SOLVE_BLOCK, warm_start=warm, tol=tol)
    return cs.fit_ai_reml(c["y"], c["x"], grm, trait, cfg)


@pytest.mark.parametrize("trait", [cs.TraitType.Binary, cs.TraitType.Quantitative])
def test_recycled_start_same_fit_fewer_launches(trait):
    c = _cohort(trait)
    zero = _fit(c, trait, cs.WARM_ZERO)
    prev = _fit(c, trait, cs.WARM_PREVIOUS)
    rec = _fit(c, trait, cs.WARM_RECYCLED)
    assert rec.iterations == prev.iterations == zero.iterations
    for r in (prev, rec):
        assert np.allclose(r.tau, zero.tau, rtol=1e-4, atol=0)
        assert np.allclose(r.alpha, zero.alpha, rtol=1e-4, atol=1e-6)
    # the probe and covariate products cost one launch more (K X joins K U) and every
    # later solve starts closer
    assert rec.n_kv_launches < prev.n_kv_launches, (rec.n_kv_launches, prev.n_kv_launches)


def test_recycled_fit_matches_oracle():
    trait = cs.TraitType.Quantitative
    c = _cohort(trait, n=1500, m=1200, seed=3)
    rec = _fit(c, trait, cs.WARM_RECYCLED, precision=cs.PREC_FP32, tol=1e-5)
    z = O.standardize(O.dosages(c["bed"], c["n"], c["g"]), c["af"][c["g"]], 0)
    o = O.fit_ai_reml(c["y"], c["x"], O.QUANTITATIVE, O.K_EXPLICIT, O.grm_explicit(z), max_iter=30,
                      tol=1e-5)
    assert np.allclose(rec.tau, o["tau"], rtol=1e-4, atol=0)


def test_learned_start_same_fit_and_reports_its_gain(capsys):
    # a quantitative trait to a tight AI-REML tolerance: several iterations, so the MLP
    # is trained on the fit's own solves and its prediction can join the start
    trait = cs.TraitType.Quantitative
    c = _cohort(trait, n=4000, m=3000, seed=11)
    zero = _fit(c, trait, cs.WARM_ZERO, tol=1e-4)
    rec = _fit(c, trait, cs.WARM_RECYCLED, tol=1e-4)
    lrn = _fit(c, trait, cs.WARM_LEARNED, tol=1e-4)
    assert lrn.iterations == zero.iterations >= 4
    assert np.allclose(lrn.tau, zero.tau, rtol=1e-4, atol=0)
    assert np.allclose(lrn.alpha, zero.alpha, rtol=1e-4, atol=1e-6)
    # against the method without the network (the recycled start): the same fit within
    # the PCG tolerance, and no more than one extra product launch per AI-REML iteration
    # (the learned start keeps the K U launch that its sketch features need)
    assert rec.iterations == lrn.iterations
    assert np.allclose(lrn.tau, rec.tau, rtol=1e-4, atol=0)
    assert lrn.n_kv_launches <= rec.n_kv_launches + lrn.iterations
    assert lrn.learned_trainings == lrn.iterations - 1
    assert 0.0 < lrn.learned_r2 <= 1.0
    with capsys.disabled():
        print(f"\n[learned start] iterations {lrn.iterations}: launches zero {zero.n_kv_launches}, "
              f"recycled {rec.n_kv_launches}, learned {lrn.n_kv_launches} "
              f"(prediction used in {lrn.learned_uses} block solves, held-out R^2 "
              f"{lrn.learned_r2:.3f}, {lrn.learned_seconds * 1e3:.1f} ms in the MLP); "
              f"PCG iterations recycled {rec.pcg_iters}, learned {lrn.pcg_iters}")


def test_diag_k_preconditioner_same_fit():
    trait = cs.TraitType.Binary
    c = _cohort(trait, n=2000, m=1500, seed=13)
    unit = _fit(c, trait, cs.WARM_PREVIOUS)
    grm = cs.OnTheFlyGrm.from_bed(c["bed"], c["n"], c["m"], c["g"], c["af"][c["g"]],
                                  precision=cs.PREC_MIXED)
    cfg = cs.AiRemlConfig(precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK,
                          warm_start=cs.WARM_PREVIOUS, precond=cs.PRECOND_DIAG_K)
    dk = cs.fit_ai_reml(c["y"], c["x"], grm, trait, cfg)
    assert np.allclose(dk.tau, unit.tau, rtol=1e-4, atol=0)
