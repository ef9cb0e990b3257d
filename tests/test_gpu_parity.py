"""GPU path vs the CPU oracle, through the C ABI (csaige_b200 is its ctypes mirror).

Integer work (allele counts, missing counts, repacking) must match bit for
bit; floating-point results are held to the tolerances written in each test.
"""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu


def _cohort(n, m, seed=7, trait=cs.api._lib.TRAIT_BINARY, n_covar=2, **kw):
    spec = cs.CohortSpec(n=n, m=m, seed=seed, trait=trait, n_covar=n_covar, **kw)
    return spec, cs.gen_bed(spec)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# ---------------------------------------------------------------- K1 counts
def test_marker_stats_fixture_bit_exact(golden_dir):
    bed = np.fromfile(golden_dir / "plink1000_500.bed", dtype=np.uint8)
    g = cs.bed_marker_stats(bed, 1000, 500)
    o = O.marker_stats(bed, 1000, 500)
    for a, b in zip(g, o):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("n", [1, 5, 16, 17, 1001, 2048])
def test_marker_stats_synthetic_bit_exact(n):
    spec, bed = _cohort(n, 97, missing_rate=0.05)
    g = cs.bed_marker_stats(bed, n, 97)
    o = O.marker_stats(bed, n, 97)
    for a, b in zip(g, o):
        assert np.array_equal(a, b)


def test_marker_stats_subset_bit_exact():
    spec, bed = _cohort(1001, 80, missing_rate=0.03)
    rng = np.random.default_rng(3)
    sidx = rng.permutation(1001)[:733]  # reordered subset, as set_sample_subset produces
    g = cs.bed_marker_stats(bed, 1001, 80, sidx)
    o = O.marker_stats(bed, 1001, 80, sidx)
    for a, b in zip(g, o):
        assert np.array_equal(a, b)


def test_generator_device_matches_host():
    torch = pytest.importorskip("torch")
    spec = cs.CohortSpec(n=3001, m=129, seed=11, cousin_frac=0.02)
    host = cs.gen_bed(spec)
    dev = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, dev.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), host)


@pytest.mark.parametrize("seed,n_vec,n", [(12345, 30, 1001), (7, 3, 17), (1, 2, 100003)])
def test_rademacher_probes_bit_exact(seed, n_vec, n):
    # the GPU draws the ChaCha8 stream block-parallel; the oracle draws it in order
    got = cs.api.rademacher_probes(seed, n_vec, n)
    want = O.probes(seed, n_vec, n)
    assert np.array_equal(got, want)


# ---------------------------------------------------------------- GRM product
def _grm_case(n=1001, m=300, seed=7, sidx=None):
    spec, bed = _cohort(n, m, seed=seed)
    af, mac, nv = O.marker_stats(bed, n, m, sidx)
    keep = np.nonzero((af >= 0.01) & (af <= 0.99))[0]
    dos = O.dosages(bed, n, keep, sidx)
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, keep, af[keep], sample_idx=sidx)
    return grm, dos, af[keep]


def test_fp32_kv_matches_oracle():
    grm, dos, afs = _grm_case()
    rng = np.random.default_rng(0)
    v = rng.standard_normal(grm.n_samples)
    got = grm.mat_vec(v)
    z32 = O.standardize(dos, afs, 1)
    want_f32 = O.grm_matvec(z32, v, 1)          # saige-rs arithmetic, 1 thread
    want_f64 = O.grm_matvec(O.standardize(dos, afs, 0), v, 0)  # FP64 oracle
    # f32 products and sums in a different order: f32 rounding level
    assert _rel(got, want_f32) < 2e-5
    assert _rel(got, want_f64) < 2e-5


def test_fp32_kv_block_and_subset():
    rng = np.random.default_rng(1)
    sidx = rng.permutation(1500)[:1100]
    grm, dos, afs = _grm_case(n=1500, m=257, seed=9, sidx=sidx)
    v = rng.standard_normal((3, grm.n_samples))
    got = grm.mat_vec(v)
    z = O.standardize(dos, afs, 0)
    for c in range(3):
        assert _rel(got[c], O.grm_matvec(z, v[c], 0)) < 2e-5


def test_kv_from_dosages_matches_bed_path():
    grm, dos, afs = _grm_case(n=640, m=200)
    g2 = cs.OnTheFlyGrm.new(dos, afs)
    v = np.random.default_rng(2).standard_normal(640)
    assert np.array_equal(grm.mat_vec(v), g2.mat_vec(v))


def test_kv_no_markers_is_zero():
    spec, bed = _cohort(100, 10)
    grm = cs.OnTheFlyGrm.from_bed(bed, 100, 10, [], [])
    assert np.all(grm.mat_vec(np.ones(100)) == 0.0)


def test_kv_dimension_mismatch_raises():
    grm, dos, afs = _grm_case(n=300, m=50)
    with pytest.raises(cs.SaigeError):
        grm.mat_vec(np.ones(299))


# ---------------------------------------------------------------- PCG
def _weights(n, seed=4):
    rng = np.random.default_rng(seed)
    mu = 1 / (1 + np.exp(-(rng.standard_normal(n) - 2)))
    return mu * (1 - mu)


def test_pcg_matches_oracle():
    grm, dos, afs = _grm_case(n=900, m=400)
    n = grm.n_samples
    w = _weights(n)
    tau = [1.0, 0.3]
    b = np.random.default_rng(5).standard_normal(n)
    z32 = O.standardize(dos, afs, 1)
    xo, ito, rso, cvo = O.pcg_sigma(O.K_OTF, z32, n, z32.shape[0], 1, w, tau, b)
    r = cs.PcgSolver(1e-5, 500).solve(grm, w, tau, b)
    assert r.converged and cvo
    assert abs(r.iterations - ito) <= 1
    assert _rel(r.x, xo) < 1e-5


def test_block_pcg_columns_match_single():
    grm, dos, afs = _grm_case(n=900, m=400)
    n = grm.n_samples
    w = _weights(n)
    tau = [1.0, 0.5]
    b = np.random.default_rng(6).standard_normal((4, n))
    solver = cs.PcgSolver(1e-5, 500)
    block = solver.solve(grm, w, tau, b)
    for c in range(4):
        single = solver.solve(grm, w, tau, b[c])
        assert block[c].iterations == single.iterations
        assert np.array_equal(block[c].x, single.x)


def test_pcg_warm_start_and_nonconvergence():
    grm, dos, afs = _grm_case(n=900, m=400)
    n = grm.n_samples
    w = _weights(n)
    tau = [1.0, 0.5]
    b = np.random.default_rng(7).standard_normal(n)
    solver = cs.PcgSolver(1e-5, 500)
    r0 = solver.solve(grm, w, tau, b)
    r1 = solver.solve(grm, w, tau, b, x0=r0.x + 1e-4)
    assert r1.converged and r1.iterations < r0.iterations
    assert _rel(r1.x, r0.x) < 1e-4
    r2 = cs.PcgSolver(1e-12, 1).solve(grm, w, tau, b)
    assert not r2.converged and r2.iterations == 1


def test_solve_mixed_model_pcg_convention():
    grm, dos, afs = _grm_case(n=700, m=300)
    n = grm.n_samples
    w = _weights(n) * 4
    tau = [1.0, 0.2]
    b = np.random.default_rng(8).standard_normal(n)
    r = cs.solve_mixed_model_pcg(tau, w, grm, b, cs.SaigePcgConfig(1e-8, 500))
    k = O.grm_explicit(O.standardize(dos, afs, 0))
    a = tau[0] * np.diag(w) + tau[1] * k
    assert r.converged
    assert np.abs(a @ r.x - b).max() / np.abs(b).max() < 1e-5


# ---------------------------------------------------------------- AI-REML
def _fit_case(trait, n=800, m=600, seed=21):
    spec, bed = _cohort(n, m, seed=seed, trait=trait, n_covar=2, prevalence=0.2, h2=0.4)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = O.marker_stats(bed, n, m)
    g, vr = O.select_markers(af, mac, nv, n)
    dos = O.dosages(bed, n, g)
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, g, af[g])
    return grm, dos, af[g], y, x


@pytest.mark.parametrize("trait", [O.BINARY, O.QUANTITATIVE])
def test_ai_reml_matches_fp64_oracle(trait):
    grm, dos, afs, y, x = _fit_case(trait)
    cfg = cs.AiRemlConfig(max_iter=6, tol=1e-5)
    r = cs.fit_ai_reml(y, x, grm, cs.TraitType(trait), cfg)
    k = O.grm_explicit(O.standardize(dos, afs, 0))
    o = O.fit_ai_reml(y, x, trait, O.K_EXPLICIT, k, max_iter=6, tol=1e-5)
    assert r.iterations == o["iterations"]
    print("tau gpu", r.tau, "oracle", o["tau"], "rel", np.abs(r.tau - o["tau"]) / o["tau"])
    assert np.all(np.abs(r.tau - o["tau"]) <= 1e-4 * np.abs(o["tau"]))
    assert np.abs(r.tau_trace - o["tau_trace"]).max() <= 1e-4 * np.abs(o["tau_trace"]).max()
    assert _rel(r.alpha, o["alpha"]) < 1e-4


def test_ai_reml_block_and_warm_start_agree():
    grm, dos, afs, y, x = _fit_case(O.BINARY, seed=23)
    base = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cs.AiRemlConfig(max_iter=5, tol=1e-5))
    blk = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary,
                         cs.AiRemlConfig(max_iter=5, tol=1e-5, solve=cs.SOLVE_BLOCK,
                                         warm_start=cs.WARM_PREVIOUS))
    print("tau single", base.tau, "block+warm", blk.tau, base.pcg_iters, blk.pcg_iters)
    assert np.all(np.abs(blk.tau - base.tau) <= 1e-4 * np.abs(base.tau))
    assert blk.n_kv_launches < base.n_kv_launches


# ---------------------------------------------------------------- diag K
@pytest.mark.parametrize("n,m,sub", [(1001, 300, False), (1500, 257, True)])
def test_grm_diag_matches_oracle(n, m, sub):
    """Get_Diagof_StdGeno (src/SAIGE_fitGLMM_fast.cpp:642-680): diag of the FP64 GRM."""
    sidx = np.random.default_rng(n).permutation(n)[: n - 137] if sub else None
    grm, dos, afs = _grm_case(n=n, m=m, sidx=sidx)
    k = O.grm_explicit(O.standardize(dos, afs, 0))
    got = grm.diag()
    assert np.abs(got - np.diag(k)).max() <= 1e-12 * np.abs(np.diag(k)).max()
