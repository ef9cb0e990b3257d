"""Variance ratio on the GPU (csaige_b200.estimate_variance_ratio, through the C ABI)
against the CPU oracle's restatement of variance_ratio.rs:87-246 / fit_null.rs:290-373.

The ratios depend on Sigma^-1 solves to the PCG tolerance (1e-5), so per-marker ratios
are compared at 1e-4 relative; the marker order and count, which follow from the
shuffle and the reference's rules, must be equal."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu

MIXED = cs.PREC_MIXED
FP32 = cs.PREC_FP32


def _setup(n=1200, m_grm=500, n_cand=120, seed=5, missing=0.01):
    spec = cs.CohortSpec(n=n, m=m_grm + n_cand, seed=seed, missing_rate=missing,
                         prevalence=0.2, h2=0.3, n_covar=2)
    bed = cs.gen_bed(spec)
    m = m_grm + n_cand
    af, mac, nv = O.marker_stats(bed, n, m)
    gidx = np.arange(m_grm)
    cidx = np.arange(m_grm, m)
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, gidx, af[gidx])
    dos_g = O.dosages(bed, n, gidx)
    z = O.standardize(dos_g, af[gidx], 0)
    cand = O.dosages(bed, n, cidx)  # NaN = missing call
    y, x = cs.gen_pheno(spec)
    fit = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cs.AiRemlConfig(max_iter=5))
    return dict(grm=grm, z=z, m_grm=m_grm, cand=cand, mac=mac[cidx], x=x, mu=fit.mu,
                w=fit.working_weights, tau=np.array(fit.tau))


@pytest.fixture(scope="module")
def case():
    return _setup()


def _oracle(c, **kw):
    return O.variance_ratio(c["cand"], c["mac"], c["mu"], c["w"], c["tau"], O.BINARY, c["x"],
                            O.K_OTF, c["z"], m=c["m_grm"], kmode=0, **kw)


@pytest.mark.parametrize("xadjust", [cs.api.VR_XADJUST_REFERENCE, cs.api.VR_XADJUST_PROJECTION])
@pytest.mark.parametrize("precision", [FP32, MIXED])
def test_all_candidates_match_oracle(case, xadjust, precision):
    c = case
    cfg = cs.VarianceRatioConfig(ratio_cv_cutoff=1e-12, xadjust=xadjust, precision=precision)
    got = cs.estimate_variance_ratio(c["grm"], c["cand"], c["mac"], c["mu"], c["w"], c["tau"],
                                     cs.TraitType.Binary, c["x"], cfg)
    want = _oracle(c, cutoff=1e-12, xadjust=xadjust)
    assert want["rc"] == 0
    assert got.n_markers_used == want["n_used"]
    assert np.array_equal(got.used_idx, want["used"])
    assert np.allclose(got.per_marker_vr, want["per_marker"], rtol=1e-4, atol=0)
    assert abs(got.variance_ratio - want["variance_ratio"]) < 1e-4 * abs(want["variance_ratio"])


def test_default_stopping_rule_matches_oracle(case):
    c = case
    got = cs.estimate_variance_ratio(c["grm"], c["cand"], c["mac"], c["mu"], c["w"], c["tau"],
                                     cs.TraitType.Binary, c["x"], cs.VarianceRatioConfig())
    want = _oracle(c)
    assert got.n_markers_used == want["n_used"] >= 30
    assert np.array_equal(got.used_idx, want["used"])
    assert abs(got.variance_ratio - want["variance_ratio"]) < 1e-4 * abs(want["variance_ratio"])


@pytest.mark.parametrize("precision", [FP32, MIXED])
def test_ratios_do_not_depend_on_block_size(case, precision):
    # each column's PCG recurrence and reductions are independent of its block
    c = case
    out = []
    for block in (7, 64):
        cfg = cs.VarianceRatioConfig(ratio_cv_cutoff=1e-12, precision=precision, block=block)
        out.append(cs.estimate_variance_ratio(c["grm"], c["cand"], c["mac"], c["mu"], c["w"],
                                              c["tau"], cs.TraitType.Binary, c["x"], cfg))
    assert np.array_equal(out[0].used_idx, out[1].used_idx)
    assert np.array_equal(out[0].per_marker_vr, out[1].per_marker_vr)
    assert out[0].n_blocks > out[1].n_blocks


def test_ratio_is_one_when_tau_g_is_zero(case):
    c = case
    w = c["mu"] * (1 - c["mu"])
    got = cs.estimate_variance_ratio(c["grm"], c["cand"], c["mac"], c["mu"], w, [1.0, 0.0],
                                     cs.TraitType.Binary, c["x"], cs.VarianceRatioConfig())
    assert got.n_markers_used == 30
    assert np.allclose(got.per_marker_vr, 1.0, rtol=0, atol=1e-9)


def test_categorical_ratios_match_oracle(case):
    c = case
    cfg = cs.VarianceRatioConfig(ratio_cv_cutoff=1e-12, use_categorical=True)
    got = cs.estimate_variance_ratio(c["grm"], c["cand"], c["mac"], c["mu"], c["w"], c["tau"],
                                     cs.TraitType.Binary, c["x"], cfg)
    want = _oracle(c, cutoff=1e-12, categorical=True)
    assert len(got.categorical_vr) == len(want["categorical"]) >= 1
    for (ua, va), (ub, vb) in zip(got.categorical_vr, want["categorical"]):
        assert ua == ub and abs(va - vb) < 1e-4 * abs(vb)


def test_no_usable_candidate_is_an_error(case):
    c = case
    with pytest.raises(cs.SaigeError):
        cs.estimate_variance_ratio(c["grm"], c["cand"][:5], np.zeros(5), c["mu"], c["w"],
                                   c["tau"], cs.TraitType.Binary, c["x"],
                                   cs.VarianceRatioConfig())


def test_fit_null_from_bed_variance_ratio_equals_the_steps():
    # the one-call pipeline (device .bed rows) against the same steps through the API
    n, m = 1500, 3000
    spec = cs.CohortSpec(n=n, m=m, seed=17, missing_rate=0.01, prevalence=0.2, h2=0.3,
                         n_covar=2)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    cfg = cs.AiRemlConfig(max_iter=4)
    fr = cs.fit_null_from_bed(bed, n, m, y, x, cs.TraitType.Binary, cfg, variance_ratio=True)
    assert fr.variance_ratio is not None and fr.m_vr > 0
    af, mac, nv = cs.bed_marker_stats(bed, n, m)
    gidx, vidx = cs.select_grm_markers(af, mac, nv, n, 0.01, 0.15, 12345)
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, gidx, af[gidx])
    fit = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg)
    assert np.array_equal(fit.tau, fr.ai_reml.tau)
    vr = cs.estimate_variance_ratio(grm, O.dosages(bed, n, vidx), mac[vidx], fit.mu,
                                    fit.working_weights, fit.tau, cs.TraitType.Binary, x)
    assert vr.n_markers_used == fr.variance_ratio.n_markers_used
    assert vr.variance_ratio == fr.variance_ratio.variance_ratio


def test_fit_null_outputs_written_and_read_back(tmp_path):
    n, m = 800, 1500
    spec = cs.CohortSpec(n=n, m=m, seed=29, prevalence=0.2, h2=0.3, n_covar=2)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    fr = cs.fit_null_from_bed(bed, n, m, y, x, cs.TraitType.Binary, cs.AiRemlConfig(max_iter=3),
                              variance_ratio=True)
    ids = [f"s{i}" for i in range(n)]
    model_path, vr_path = cs.save_fit_null(tmp_path / "example", fr, cs.TraitType.Binary, ids,
                                           y, x)
    mdl = cs.load_model(model_path)
    assert np.array_equal(mdl.tau, fr.ai_reml.tau)
    assert mdl.variance_ratio.variance_ratio == fr.variance_ratio.variance_ratio
    assert open(vr_path).read().endswith(" null 1\n")


@pytest.mark.parametrize("subset,trait", [(False, cs.TraitType.Binary),
                                           (True, cs.TraitType.Binary),
                                           (True, cs.TraitType.Quantitative)])
def test_pinned_upload_path_gives_the_same_fit(subset, trait):
    # from pinned host memory a MIXED fit builds its GRM while the .bed streams in: the
    # rows are all QC-passing markers, the variance-ratio candidates kept with zero 2p
    # and 1/s; the products are exact integers, so the fit and the ratio must equal
    # those of the steps on pageable memory (GRM markers only) bit for bit
    import torch
    n, m = 1500, 2500
    spec = cs.CohortSpec(n=n, m=m, seed=31, missing_rate=0.02, prevalence=0.2, h2=0.3, n_covar=2,
                         trait=trait)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    sidx = None
    if subset:
        sidx = np.sort(np.random.default_rng(3).choice(n, 1201, replace=False))
        y, x = y[sidx], x[sidx]
    pinned = torch.empty(bed.size, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = bed
    cfg = cs.AiRemlConfig(max_iter=4, precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK,
                          warm_start=cs.WARM_RECYCLED)
    # a MAF filter that drops markers in every chunk
    kw = dict(sample_idx=sidx, min_maf=0.05, variance_ratio=True)
    a = cs.fit_null_from_bed(bed, n, m, y, x, trait, cfg, **kw)
    b = cs.fit_null_from_bed(pinned.numpy(), n, m, y, x, trait, cfg, **kw)
    assert 0 < a.m_grm < m - a.m_vr
    assert (a.m_grm, a.m_vr) == (b.m_grm, b.m_vr)
    assert np.array_equal(a.ai_reml.tau, b.ai_reml.tau)
    assert np.array_equal(a.ai_reml.alpha, b.ai_reml.alpha)
    assert a.variance_ratio.variance_ratio == b.variance_ratio.variance_ratio


@pytest.mark.parametrize("concurrent,tune,prec", [(True, False, "mixed"), (False, False, "mixed"),
                                                  (True, True, "mixed"), (True, False, "fp32")])
def test_sub_cohort_fits_equal_their_own_fits(concurrent, tune, prec, monkeypatch):
    # fit_null::run per sub-cohort of one .bed, concurrently on threads and streams; with
    # tune, the ring-shape autotuner runs on every launch size, so the concurrent fits'
    # products share its per-key candidate state (results are the same for every shape)
    if tune:
        monkeypatch.setenv("SAIGE_TC_AUTOTUNE", "2")
    n, m = 3000, 2000
    spec = cs.CohortSpec(n=n, m=m, seed=37, missing_rate=0.01, prevalence=0.3, h2=0.3, n_covar=2)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    rng = np.random.default_rng(5)
    cohorts = []
    for size in (700, 1300, 2203):
        idx = np.sort(rng.choice(n, size, replace=False))
        cohorts.append((idx, y[idx], x[idx]))
    # every sample, in shuffled order (the concurrent path counts all cohorts in one
    # launch per marker chunk: unsorted indices and a ragged last word included)
    idx = rng.permutation(n)
    cohorts.append((idx, y[idx], x[idx]))
    # MIXED: the concurrent call builds every cohort's rows under the streamed upload
    # (all QC-passing markers, the variance-ratio ones kept in place with zero metadata);
    # FP32: one shared gather of the GRM markers after all counts
    cfg = cs.AiRemlConfig(max_iter=6, solve=cs.SOLVE_BLOCK, warm_start=cs.WARM_RECYCLED,
                          precision=cs.PREC_MIXED if prec == "mixed" else cs.PREC_FP32)
    res, wall = cs.fit_null_cohorts(bed, n, m, cohorts, cs.TraitType.Binary, cfg,
                                    concurrent=concurrent)
    assert wall > 0 and len(res) == 4
    for (idx, yc, xc), r in zip(cohorts, res):
        one = cs.fit_null_from_bed(bed, n, m, yc, xc, cs.TraitType.Binary, cfg, sample_idx=idx)
        assert r.m_grm == one.m_grm
        assert np.array_equal(r.tau, one.ai_reml.tau)
        assert np.array_equal(r.alpha, one.ai_reml.alpha)


def test_concurrent_sub_cohort_fits_are_bit_identical_to_sequential():
    # Eight mid-size cohorts fitted concurrently (their tensor-core launches share the
    # SMs with each other's vector kernels, which changes the pipeline timing) must give
    # exactly the sequential fits: every product is an exact integer sum, so any
    # difference is a pipeline race.  Block PCG from zero starts runs the most
    # 42-column products (pass B on a three-stage load ring).
    n, m = 60_000, 40_000
    spec = cs.CohortSpec(n=n, m=m, seed=91, missing_rate=0.01, prevalence=0.1, h2=0.2, n_covar=4)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    rng = np.random.default_rng(17)
    cohorts = []
    for size in (8_000, 11_000, 15_000, 19_000, 23_000, 27_000, 31_000, 36_000):
        idx = np.sort(rng.choice(n, size, replace=False))
        cohorts.append((idx, y[idx], x[idx]))
    cfg = cs.AiRemlConfig(max_iter=8, tol=1e-5, precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK,
                          warm_start=cs.WARM_ZERO)
    seq, _ = cs.fit_null_cohorts(bed, n, m, cohorts, cs.TraitType.Binary, cfg, concurrent=False)
    for _ in range(3):
        con, _ = cs.fit_null_cohorts(bed, n, m, cohorts, cs.TraitType.Binary, cfg, concurrent=True)
        for a, b in zip(seq, con):
            assert a.m_grm == b.m_grm
            assert np.array_equal(a.tau, b.tau)
            assert np.array_equal(a.alpha, b.alpha)


@pytest.mark.parametrize("prec", ["mixed", "fp32"])
def test_more_cohorts_than_one_gather_launch_holds(prec):
    # 35 cohorts: the concurrent call gathers their rows in launches of at most 32 cohorts
    # (the cohorts' outputs ride in the launch parameters), so two launches per chunk
    n, m = 3000, 1500
    spec = cs.CohortSpec(n=n, m=m, seed=53, missing_rate=0.01, prevalence=0.3, h2=0.3, n_covar=2)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    rng = np.random.default_rng(9)
    cohorts = []
    for size in rng.integers(400, 900, 35):
        idx = np.sort(rng.choice(n, int(size), replace=False))
        cohorts.append((idx, y[idx], x[idx]))
    cfg = cs.AiRemlConfig(max_iter=3, solve=cs.SOLVE_BLOCK, warm_start=cs.WARM_RECYCLED,
                          precision=cs.PREC_MIXED if prec == "mixed" else cs.PREC_FP32)
    seq, _ = cs.fit_null_cohorts(bed, n, m, cohorts, cs.TraitType.Binary, cfg, concurrent=False)
    con, _ = cs.fit_null_cohorts(bed, n, m, cohorts, cs.TraitType.Binary, cfg, concurrent=True)
    assert len(con) == 35
    for a, b in zip(seq, con):
        assert a.m_grm == b.m_grm
        assert np.array_equal(a.tau, b.tau)
        assert np.array_equal(a.alpha, b.alpha)
