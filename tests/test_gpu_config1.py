"""fit-null parity on the reference's own CPU-scale cohort, GPU against the FP64 oracle.

The cohort is the plain fit-null case: N = 2,000 samples, M = 5,000 bed markers,
MAF ~ U(0.01, 0.5), HWE genotypes, 1 % missing calls at random, 10 % of the
samples in sibling pairs, a binary trait at ~10 % prevalence from
logit(b0 + 0.3 N(0,1) + 0.2 Bernoulli(0.5) + polygenic score, h2 = 0.2),
30 Rademacher probes, PCG tolerance 1e-5, the Jacobi preconditioner.

The oracle fits with the exact FP64 GRM (oracle/oracle.c `orc_fit_ai_reml`,
restating saige-core/src/glmm/ai_reml.rs:86-427).  Every GPU configuration is
held to the same bar:

* tau within 1e-4 relative of the oracle's (the AI-REML tolerance of the
  comparison is the AiRemlConfig default 0.02 and the fit-null command's 1e-5,
  saige-cli/src/commands/fit_null.rs:74-80);
* alpha within 1e-4 relative (max-norm);
* Sigma^-1 y from the library's PCG at the fit's own tau and W has a true
  residual ||y - Sigma x|| / ||y|| of at most 1.05e-5 against the FP64 Sigma —
  the PCG tolerance 1e-5 plus the product's own rounding — and is within 1e-4 of
  the exact solution.
"""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu

TAU_REL = 1e-4
ALPHA_REL = 1e-4
RESID_REL = 1.05e-5   # PCG tolerance 1e-5 plus the product's rounding
X_REL = 1e-4


@pytest.fixture(scope="module")
def cohort():
    spec = cs.CohortSpec()  # the defaults are this cohort, seed 12345
    assert (spec.n, spec.m, spec.missing_rate, spec.sib_frac, spec.prevalence) == \
        (2000, 5000, 0.01, 0.10, 0.10)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = O.marker_stats(bed, spec.n, spec.m)
    g, _ = O.select_markers(af, mac, nv, spec.n)
    k = O.grm_explicit(O.standardize(O.dosages(bed, spec.n, g), af[g], 0))
    oracle = {tol: O.fit_ai_reml(y, x, O.BINARY, O.K_EXPLICIT, k, max_iter=30, tol=tol)
              for tol in (0.02, 1e-5)}
    return dict(spec=spec, bed=bed, y=y, x=x, af=af, g=g, k=k, oracle=oracle)


CONFIGS = {
    # the reference's strategy: FP32 products, one PCG per right-hand side, zero starts
    "fp32_single": dict(precision=cs.PREC_FP32, solve=cs.SOLVE_SINGLE, warm_start=cs.WARM_ZERO),
    "mixed_single": dict(precision=cs.PREC_MIXED, solve=cs.SOLVE_SINGLE,
                         warm_start=cs.WARM_ZERO),
    # the benchmark's fast configuration
    "mixed_block_recycled": dict(precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK,
                                 warm_start=cs.WARM_RECYCLED),
    "fp32_block_recycled": dict(precision=cs.PREC_FP32, solve=cs.SOLVE_BLOCK,
                                warm_start=cs.WARM_RECYCLED),
}


def _grm(c, precision):
    s = c["spec"]
    return cs.OnTheFlyGrm.from_bed(c["bed"], s.n, s.m, c["g"], c["af"][c["g"]],
                                   precision=precision)


def _sigma(c, tau, w):
    return tau[0] * np.diag(1.0 / np.maximum(w, 1e-30)) + tau[1] * c["k"]


@pytest.mark.parametrize("tol", [0.02, 1e-5])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_fit_matches_fp64_oracle(cohort, name, tol, capsys):
    c = cohort
    o = c["oracle"][tol]
    kw = CONFIGS[name]
    grm = _grm(c, kw["precision"])
    r = cs.fit_ai_reml(c["y"], c["x"], grm, cs.TraitType.Binary,
                       cs.AiRemlConfig(max_iter=30, tol=tol, **kw))
    tau_rel = np.abs(r.tau - o["tau"]) / np.abs(o["tau"])
    a_rel = np.abs(r.alpha - o["alpha"]).max() / np.abs(o["alpha"]).max()
    # Sigma^-1 y with the library's PCG at the fit's own tau and W
    sol = cs.PcgSolver(1e-5, 500).solve(grm, r.working_weights, r.tau, c["y"])
    sig = _sigma(c, r.tau, r.working_weights)
    resid = np.linalg.norm(c["y"] - sig @ sol.x) / np.linalg.norm(c["y"])
    exact = np.linalg.solve(sig, c["y"])
    x_rel = np.linalg.norm(sol.x - exact) / np.linalg.norm(exact)
    with capsys.disabled():
        print(f"\n[config 1 {name} tol {tol:g}] tau {r.tau[1]:.9f} oracle {o['tau'][1]:.9f} "
              f"rel {tau_rel[1]:.2e}; alpha rel {a_rel:.2e}; AI-REML iterations {r.iterations} "
              f"(oracle {o['iterations']}); Sigma^-1 y residual {resid:.2e}, error {x_rel:.2e}; "
              f"launches {r.n_kv_launches}, PCG iterations {r.pcg_iters}")
    assert r.converged and o["converged"]
    assert np.all(tau_rel <= TAU_REL), tau_rel
    assert a_rel <= ALPHA_REL, a_rel
    assert sol.converged
    assert resid <= RESID_REL, resid
    assert x_rel <= X_REL, x_rel
    if kw["warm_start"] == cs.WARM_ZERO:
        # the reference's solve order and zero starts: the same tau trajectory
        assert r.iterations == o["iterations"]
        assert np.abs(r.tau_trace - o["tau_trace"]).max() <= TAU_REL * np.abs(o["tau_trace"]).max()


@pytest.mark.parametrize("precision", [cs.PREC_FP32, cs.PREC_MIXED])
def test_block_solve_of_the_fit_rhs_to_pcg_tolerance(cohort, precision):
    """[y, X, probes] in one block PCG at the oracle's final tau and W: every column
    reaches the PCG tolerance against the FP64 Sigma."""
    c = cohort
    o = c["oracle"][1e-5]
    n = c["spec"].n
    rhs = np.vstack([c["y"][None, :], c["x"].T, O.probes(12345, 30, n)])
    grm = _grm(c, precision)
    res = cs.PcgSolver(1e-5, 500).solve(grm, o["w"], o["tau"], rhs, precision=precision)
    sig = _sigma(c, o["tau"], o["w"])
    for col, r in enumerate(res):
        b = rhs[col]
        resid = np.linalg.norm(b - sig @ r.x) / max(np.linalg.norm(b), 1.0)
        assert r.converged, col
        assert resid <= RESID_REL, (col, resid)


@pytest.fixture(scope="module")
def cohort_quant():
    """The same CPU-scale cohort with a quantitative trait (4 N(0,1) covariates,
    h2 = 0.3, Gaussian noise): tau0 is estimated too, with the W^-1 AI solve
    (ai_reml.rs:281-306)."""
    spec = cs.CohortSpec(trait=cs.TraitType.Quantitative, n_covar=4, h2=0.3)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = O.marker_stats(bed, spec.n, spec.m)
    g, _ = O.select_markers(af, mac, nv, spec.n)
    k = O.grm_explicit(O.standardize(O.dosages(bed, spec.n, g), af[g], 0))
    oracle = {tol: O.fit_ai_reml(y, x, O.QUANTITATIVE, O.K_EXPLICIT, k, max_iter=30, tol=tol)
              for tol in (0.02, 1e-5)}
    return dict(spec=spec, bed=bed, y=y, x=x, af=af, g=g, k=k, oracle=oracle)


@pytest.mark.parametrize("tol", [0.02, 1e-5])
@pytest.mark.parametrize("name", list(CONFIGS))
def test_quantitative_fit_matches_fp64_oracle(cohort_quant, name, tol, capsys):
    c = cohort_quant
    o = c["oracle"][tol]
    kw = CONFIGS[name]
    grm = _grm(c, kw["precision"])
    r = cs.fit_ai_reml(c["y"], c["x"], grm, cs.TraitType.Quantitative,
                       cs.AiRemlConfig(max_iter=30, tol=tol, **kw))
    tau_rel = np.abs(r.tau - o["tau"]) / np.abs(o["tau"])
    a_rel = np.abs(r.alpha - o["alpha"]).max() / np.abs(o["alpha"]).max()
    sol = cs.PcgSolver(1e-5, 500).solve(grm, r.working_weights, r.tau, c["y"])
    sig = _sigma(c, r.tau, r.working_weights)
    resid = np.linalg.norm(c["y"] - sig @ sol.x) / np.linalg.norm(c["y"])
    with capsys.disabled():
        print(f"\n[config 1 quantitative {name} tol {tol:g}] tau {r.tau} oracle {o['tau']} "
              f"rel {tau_rel.max():.2e}; alpha rel {a_rel:.2e}; AI-REML iterations "
              f"{r.iterations} (oracle {o['iterations']}); residual {resid:.2e}; "
              f"launches {r.n_kv_launches}")
    assert r.converged and o["converged"]
    assert np.all(tau_rel <= TAU_REL), tau_rel
    assert a_rel <= ALPHA_REL, a_rel
    assert sol.converged and resid <= RESID_REL, resid
    if kw["warm_start"] == cs.WARM_ZERO:
        assert r.iterations == o["iterations"]
