"""Variance-ratio estimation (variance_ratio.rs:87-246, fit_null.rs:290-373): the
oracle's restatement and the library's host-side pieces, on the CPU."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O


@pytest.mark.parametrize("seed,length", [(12345, 997), (7, 1), (1, 2), (99, 0), (3, 40)])
def test_marker_order_matches_oracle_shuffle(seed, length):
    got = cs.vr_marker_order(seed, length)
    want = O.shuffled_indices(seed, length)
    assert np.array_equal(got, want)
    assert np.array_equal(np.sort(got), np.arange(length))  # a permutation


def test_shuffle_depends_on_seed():
    assert not np.array_equal(O.shuffled_indices(1, 50), O.shuffled_indices(2, 50))


def test_gen_range_u32_in_bounds():
    r = O.ChaChaRng()
    O.L.orc_chacha_seed_from_u64(O.C.byref(r), 5, 8)
    vals = [O.L.orc_rng_gen_range_u32(O.C.byref(r), 0, 7) for _ in range(2000)]
    assert min(vals) == 0 and max(vals) == 6
    assert all(0 <= v < 7 for v in vals)


def _cohort(n, n_cand, seed=3, missing=0.0):
    rng = np.random.default_rng(seed)
    p_af = rng.uniform(0.05, 0.5, n_cand)
    d = rng.binomial(2, p_af[:, None], size=(n_cand, n)).astype(float)
    if missing:
        d[rng.random(d.shape) < missing] = np.nan
    s = np.nansum(d, axis=1)
    nv = np.sum(~np.isnan(d), axis=1)
    mac = np.minimum(s, 2 * nv - s)
    x = np.column_stack([np.ones(n), rng.standard_normal(n), rng.integers(0, 2, n)])
    mu = 1.0 / (1.0 + np.exp(-rng.normal(-1.5, 0.5, n)))
    return d, mac, x, mu


@pytest.mark.parametrize("trait", [O.BINARY, O.QUANTITATIVE])
def test_oracle_ratio_is_one_when_tau_g_is_zero(trait):
    # Sigma = tau0 diag(1/w); with w = mu(1-mu) (binary) or 1 (quantitative) the exact and
    # the approximate variances coincide: every ratio is 1 and the CV test stops at 30.
    n = 400
    d, mac, x, mu = _cohort(n, 60)
    w = mu * (1 - mu) if trait == O.BINARY else np.ones(n)
    r = O.variance_ratio(d, mac, mu, w, [1.0, 0.0], trait, x, O.K_IDENTITY, None)
    assert r["rc"] == 0
    assert r["n_used"] == 30
    assert np.allclose(r["per_marker"], 1.0, rtol=0, atol=1e-9)


def test_oracle_single_covariate_layouts_agree():
    # with p = 1 the reference's column-major read of the p x n array is the projection itself
    n = 300
    d, mac, x, mu = _cohort(n, 40)
    w = mu * (1 - mu)
    k = np.eye(n) * 0.6 + 0.4 / n
    a = O.variance_ratio(d, mac, mu, w, [1.0, 0.3], O.BINARY, x[:, :1], O.K_EXPLICIT, k,
                         xadjust=0, cutoff=1e-12)
    b = O.variance_ratio(d, mac, mu, w, [1.0, 0.3], O.BINARY, x[:, :1], O.K_EXPLICIT, k,
                         xadjust=1, cutoff=1e-12)
    assert np.allclose(a["per_marker"], b["per_marker"], rtol=1e-12, atol=0)


def test_oracle_missing_calls_give_finite_ratios():
    n = 300
    d, mac, x, mu = _cohort(n, 40, missing=0.02)
    w = mu * (1 - mu)
    k = np.eye(n) * 0.6 + 0.4 / n
    r = O.variance_ratio(d, mac, mu, w, [1.0, 0.3], O.BINARY, x, O.K_EXPLICIT, k, cutoff=1e-12)
    assert r["rc"] == 0 and r["n_used"] == 40
    assert np.all(np.isfinite(r["per_marker"]))


def test_oracle_no_usable_marker():
    n = 200
    d, mac, x, mu = _cohort(n, 10)
    r = O.variance_ratio(d, np.zeros(10), mu, mu * (1 - mu), [1.0, 0.3], O.BINARY, x,
                         O.K_IDENTITY, None)
    assert r["rc"] == 1 and r["n_used"] == 0


def test_variance_ratio_file_format(tmp_path):
    # variance_ratio.rs:306-338 and the R output example_binary.varianceRatio.txt
    res = cs.VarianceRatioResult(0.94022084164312, [], 30, np.zeros(0), np.zeros(0, np.int64))
    f = tmp_path / "a.varianceRatio.txt"
    cs.write_variance_ratio_file(res, f)
    assert f.read_text() == "0.94022084164312 null 1\n"
    res2 = cs.VarianceRatioResult(0.9, [(10.5, 0.8), (float("inf"), 1.0)], 30, np.zeros(0),
                                  np.zeros(0, np.int64))
    cs.write_variance_ratio_file(res2, f)
    assert f.read_text() == "0.8 null 1\n1 null 2\n"
