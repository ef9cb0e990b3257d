"""MIXED-precision (tcgen05 kind::i8) GRM product, PCG and AI-REML on the GPU.

The integer tensor-core arithmetic is checked bit for bit against a CPU model
of the same quantised arithmetic; the quantisation error is then bounded
against the FP64 oracle."""
import numpy as np
import pytest

import csaige_b200 as cs
import mixed_model as MM
import oracle_ffi as O

pytestmark = pytest.mark.gpu
MIXED = cs.PREC_MIXED


def _case(n, m, seed=7, sidx=None, miss=0.03):
    spec = cs.CohortSpec(n=n, m=m, seed=seed, missing_rate=miss)
    bed = cs.gen_bed(spec)
    af, mac, nv = O.marker_stats(bed, n, m, sidx)
    keep = np.nonzero((af >= 0.01) & (af <= 0.99))[0]
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, keep, af[keep], sample_idx=sidx, precision=MIXED)
    return grm, bed, keep, af[keep]


@pytest.mark.parametrize("n,m,r", [(1001, 300, 1), (700, 129, 5), (2048, 256, 3)])
def test_mixed_kv_bit_exact_vs_model(n, m, r):
    grm, bed, keep, afs = _case(n, m)
    v = np.random.default_rng(n + r).standard_normal((r, grm.n_samples))
    got = grm.mat_vec(v)
    want = MM.kv(MM.codes(bed, n, keep), afs, v.T).T
    assert np.array_equal(got, want)


def test_mixed_kv_subset_bit_exact():
    rng = np.random.default_rng(9)
    sidx = rng.permutation(1500)[:1111]
    grm, bed, keep, afs = _case(1500, 200, sidx=sidx)
    v = rng.standard_normal((2, grm.n_samples))
    got = grm.mat_vec(v)
    want = MM.kv(MM.codes(bed, 1500, keep, sidx), afs, v.T).T
    assert np.array_equal(got, want)


def test_mixed_kv_more_columns_than_one_launch():
    grm, bed, keep, afs = _case(513, 140)
    v = np.random.default_rng(1).standard_normal((70, grm.n_samples))
    got = grm.mat_vec(v)
    want = MM.kv(MM.codes(bed, 513, keep), afs, v.T).T
    assert np.array_equal(got, want)


def test_mixed_kv_accuracy_vs_fp64_oracle():
    grm, bed, keep, afs = _case(3000, 800)
    v = np.random.default_rng(2).standard_normal((4, grm.n_samples))
    z = O.standardize(O.dosages(bed, 3000, keep), afs, 0)
    got = grm.mat_vec(v)
    for c in range(4):
        want = O.grm_matvec(z, v[c], 0)
        err = np.abs(got[c] - want).max() / np.abs(want).max()
        assert err < 5e-7, err


def test_mixed_pcg_matches_fp64_oracle():
    grm, bed, keep, afs = _case(1200, 500)
    n = grm.n_samples
    rng = np.random.default_rng(3)
    mu = 1 / (1 + np.exp(-(rng.standard_normal(n) - 2)))
    w = mu * (1 - mu)
    tau = [1.0, 0.4]
    b = rng.standard_normal((3, n))
    k = O.grm_explicit(O.standardize(O.dosages(bed, 1200, keep), afs, 0))
    res = cs.PcgSolver(1e-6, 500).solve(grm, w, tau, b, precision=MIXED)
    for c in range(3):
        xo, ito, rso, cvo = O.pcg_sigma(O.K_EXPLICIT, k, n, 0, 0, w, tau, b[c], tol=1e-6)
        assert res[c].converged and abs(res[c].iterations - ito) <= 1
        assert np.abs(res[c].x - xo).max() / np.abs(xo).max() < 1e-5


@pytest.mark.parametrize("trait", [O.BINARY, O.QUANTITATIVE])
def test_mixed_ai_reml_tau_within_1e4_of_fp64_oracle(trait):
    spec = cs.CohortSpec(n=800, m=600, seed=21, trait=trait, n_covar=2, prevalence=0.2, h2=0.4)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = O.marker_stats(bed, 800, 600)
    g, _ = O.select_markers(af, mac, nv, 800)
    grm = cs.OnTheFlyGrm.from_bed(bed, 800, 600, g, af[g], precision=MIXED)
    k = O.grm_explicit(O.standardize(O.dosages(bed, 800, g), af[g], 0))
    o = O.fit_ai_reml(y, x, trait, O.K_EXPLICIT, k, max_iter=8, tol=1e-5)
    for solve, warm in [(cs.SOLVE_SINGLE, cs.WARM_ZERO), (cs.SOLVE_BLOCK, cs.WARM_PREVIOUS)]:
        cfg = cs.AiRemlConfig(max_iter=8, tol=1e-5, precision=MIXED, solve=solve, warm_start=warm)
        r = cs.fit_ai_reml(y, x, grm, cs.TraitType(trait), cfg)
        rel = np.abs(r.tau - o["tau"]) / np.abs(o["tau"])
        print("solve", solve, "warm", warm, "tau", r.tau, "oracle", o["tau"], "rel", rel,
              "iters", r.iterations, o["iterations"])
        if warm == cs.WARM_ZERO:
            # the reference's solve order and starts: the same trajectory
            assert r.iterations == o["iterations"]
        # warm starts change where each solve stops inside the PCG tolerance, so the
        # tau trajectory differs at that level and the iteration count may differ
        assert r.converged and np.all(rel <= 1e-4)


def test_large_blocks_reused_from_cache_give_same_products():
    # genotypes 602 MB and two 602 MB tile copies: above the 256 MiB cache threshold
    torch = pytest.importorskip("torch")
    n, m = 200000, 12000
    spec = cs.CohortSpec(n=n, m=m, seed=21)
    bed = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, bed.data_ptr())
    torch.cuda.synchronize()
    af = np.linspace(0.05, 0.5, m)
    v = np.random.default_rng(4).standard_normal((2, n))
    outs = []
    for rep in range(3):
        if rep == 2:
            cs.api.release_cached_memory()
        grm = cs.OnTheFlyGrm.from_bed_dev(bed.data_ptr(), spec.bed_len, n, m, np.arange(m), af,
                                          precision=MIXED)
        outs.append(grm.mat_vec(v))
        grm.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def test_autotuned_ring_shapes_give_identical_products(monkeypatch):
    # the ring shape changes only the speed of the exact-integer product
    n, m = 3000, 2600
    spec = cs.CohortSpec(n=n, m=m, seed=41, missing_rate=0.01)
    bed = cs.gen_bed(spec)
    af, mac, nv = cs.bed_marker_stats(bed, n, m)
    g, _ = cs.select_grm_markers(af, mac, nv, n)
    v = np.random.default_rng(3).standard_normal((37, n))
    monkeypatch.setenv("SAIGE_TC_AUTOTUNE", "0")
    fixed = cs.OnTheFlyGrm.from_bed(bed, n, m, g, af[g], precision=cs.PREC_MIXED).mat_vec(v)
    monkeypatch.setenv("SAIGE_TC_AUTOTUNE", "2")  # tune this small size too
    before = int(cs.api.LIB.saige_tc_autotune_trials())
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, g, af[g], precision=cs.PREC_MIXED)
    # each product runs the next candidate shape of both passes' keys until all have
    # run (at most 6 per key), then the fastest: every product is the same
    for it in range(8):
        assert np.array_equal(grm.mat_vec(v), fixed), it
    assert int(cs.api.LIB.saige_tc_autotune_trials()) > before


@pytest.mark.parametrize("lists", ["2", "0"])
@pytest.mark.parametrize("n,m,sub,miss", [(1001, 300, False, 0.02), (17000, 4300, False, 0.02),
                                          (4500, 700, True, 0.02), (3000, 900, False, 0.0),
                                          (3000, 900, False, 0.06)])
def test_single_column_cuda_core_path_equals_tensor_core_path(monkeypatch, n, m, sub, miss, lists):
    # one active column runs both passes with dp4a on the CUDA cores: the same exact
    # integer sums and the same FP64 epilogue, so every bit agrees with the tensor-core
    # passes (SAIGE_SC=0) and with the CPU model; the sizes cross the staging chunks
    # (1024 sample words in pass A, 2048 markers in pass B, 8192 values of the lists' sums).
    # With the lists (SAIGE_SR_LISTS=2: built at the handle's first one-column product)
    # the sums over missing calls come from the per-block segments of missing calls; over
    # 3 % missing the lists are declined and the dense flag sums stay, as they do with
    # SAIGE_SR_LISTS=0.
    monkeypatch.setenv("SAIGE_SR_LISTS", lists)
    rng = np.random.default_rng(n + m)
    sidx = rng.permutation(n)[: n - 37] if sub else None
    grm, bed, keep, afs = _case(n, m, sidx=sidx, miss=miss)
    codes = MM.codes(bed, n, keep, sidx)
    v = rng.standard_normal((1, grm.n_samples))
    before = grm.stats()
    got = grm.mat_vec(v)
    st = grm.stats()
    assert st["sc_launches"] == before["sc_launches"] + 1
    listed = lists == "2" and miss <= 0.02
    assert st["sc_list_launches"] == before["sc_list_launches"] + int(listed)
    assert st["missing_listed"] == (int((codes == 1).sum()) if listed else -1)
    monkeypatch.setenv("SAIGE_SC", "0")
    tc = grm.mat_vec(v)
    assert grm.stats()["sc_launches"] == before["sc_launches"] + 1
    assert np.array_equal(got, tc)
    want = MM.kv(codes, afs, v.T).T
    assert np.array_equal(got, want)


def test_missing_lists_built_in_a_handles_second_fit(monkeypatch):
    # by default a handle's first AI-REML fit keeps the dense flag sums and its second fit
    # builds the missing-call lists at its first one-column product: the products are the
    # same integers, so the two fits agree to the bit
    monkeypatch.delenv("SAIGE_SR_LISTS", raising=False)
    spec = cs.CohortSpec(n=3000, m=1500, seed=31)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = cs.bed_marker_stats(bed, spec.n, spec.m)
    g, _ = cs.select_grm_markers(af, mac, nv, spec.n)
    grm = cs.OnTheFlyGrm.from_bed(bed, spec.n, spec.m, g, af[g], precision=MIXED)
    cfg = cs.AiRemlConfig(max_iter=30, tol=1e-5, precision=MIXED, solve=cs.SOLVE_BLOCK,
                          warm_start=cs.WARM_RECYCLED)
    r1 = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg)
    st = grm.stats()
    assert st["sc_launches"] > 0 and st["missing_listed"] == -1 and st["sc_list_launches"] == 0
    r2 = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg)
    st = grm.stats()
    assert st["missing_listed"] > 0 and st["sc_list_launches"] > 0
    assert np.array_equal(r1.tau, r2.tau) and np.array_equal(r1.alpha, r2.alpha)
