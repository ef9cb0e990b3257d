"""The CPU oracle against the reference's own golden vectors and known answers.

These pin the oracle before it is trusted as the checker of the GPU path.
"""
import json

import numpy as np
import pytest

import oracle_ffi as O


def test_decode_known_answers(golden_dir):
    # saige-geno/src/plink.rs:288-303
    kat = json.loads((golden_dir / "decode_kat.json").read_text())
    for byte, off, want in kat["single"]:
        got = O.decode(byte, off)
        assert (np.isnan(got) if want is None else got == want)
    for off, want in kat["offsets"]:
        got = O.decode(kat["byte"], off)
        assert (np.isnan(got) if want is None else got == want)


def _frq(golden_dir):
    rows = [l.split() for l in (golden_dir / "plink1000_500.frq").read_text().splitlines()[1:]]
    return np.array([float(r[4]) for r in rows]), np.array([int(r[5]) for r in rows])


def test_marker_stats_match_plink_frq(golden_dir):
    # PLINK's .frq MAF (4 significant digits) and NCHROBS for the fixture
    bed = np.fromfile(golden_dir / "plink1000_500.bed", dtype=np.uint8)
    maf_ref, nchrobs = _frq(golden_dir)
    af, mac, nv = O.marker_stats(bed, 1000, maf_ref.size)
    maf = np.minimum(af, 1 - af)
    assert np.array_equal(2 * nv, nchrobs)
    assert all(float(f"{a:.4g}") == b for a, b in zip(maf, maf_ref))
    # mac = min(sum, 2n - sum) is an exact integer
    assert np.array_equal(mac, np.round(mac))


def test_marker_stats_rejects_bad_bed(golden_dir):
    bed = np.fromfile(golden_dir / "plink1000_500.bed", dtype=np.uint8)
    bad = bed.copy()
    bad[0] = 0
    with pytest.raises(ValueError):
        O.marker_stats(bad, 1000, 500)
    with pytest.raises(ValueError):
        O.marker_stats(bed[:-1], 1000, 500)


def test_chacha_block_matches_independent_chacha20():
    # The ChaCha core (8 rounds for ChaCha8Rng) is the ChaCha20 block function
    # with fewer double rounds; pin it against OpenSSL's ChaCha20.
    Cipher = pytest.importorskip("cryptography.hazmat.primitives.ciphers")
    key = bytes(range(32))
    kw = np.frombuffer(key, dtype="<u4")
    for ctr in (0, 1, 7):
        mine = O.chacha_block(kw, ctr, 0, 20).astype("<u4").tobytes()
        nonce = ctr.to_bytes(4, "little") + b"\x00" * 12
        enc = Cipher.Cipher(Cipher.algorithms.ChaCha20(key, nonce), mode=None).encryptor()
        assert mine == enc.update(b"\x00" * 64)


def test_rng_stream_properties():
    # contiguous u32 stream across the 4-block buffer; gen_range stays in range
    s = O.chacha8_u32_stream(12345, 200)
    assert len(set(s.tolist())) > 190
    r = O.gen_range_u64(12345, 0, 37, 2000)
    assert r.min() == 0 and r.max() == 36
    pr = O.probes(12345, 3, 1000)
    assert set(np.unique(pr)) == {-1.0, 1.0}
    assert abs(pr.mean()) < 0.1


def test_pcg_known_answers():
    # decomposition.rs:469-500
    x, it, rs, conv = O.pcg_dense(np.eye(3), [1.0, 2.0, 3.0])
    assert conv and np.allclose(x, [1, 2, 3], atol=1e-10)
    a = np.array([[4.0, 2, 1], [2, 5, 3], [1, 3, 6]])
    x, it, rs, conv = O.pcg_dense(a, [1.0, 2.0, 3.0], tol=1e-10, max_iter=1000)
    assert conv and np.abs(a @ x - [1, 2, 3]).max() < 1e-8


def test_sigma_pcg_identity_grm():
    # pcg.rs:202-222 (tau=[1,0.1], w=1, identity GRM): x = b/1.1 to 1e-5
    b = np.array([1.0, 2, 3, 4, 5])
    x, it, rs, conv = O.pcg_sigma(O.K_IDENTITY, None, 5, 0, 0, np.ones(5), [1.0, 0.1], b)
    assert conv and np.abs(x - b / 1.1).max() < 1e-5


def test_cholesky_known_answers():
    # decomposition.rs:371-407
    l = O.cholesky(np.array([[4.0, 2], [2, 3]]))
    assert np.allclose(l, [[2, 0], [1, np.sqrt(2)]], atol=1e-10)
    a = np.array([[4.0, 2, 1], [2, 5, 3], [1, 3, 6]])
    x = O.chol_solve(O.cholesky(a), [1.0, 2, 3])
    assert np.abs(a @ x - [1, 2, 3]).max() < 1e-10
    assert O.cholesky(np.array([[1.0, 3], [3, 1]])) is None


def test_links_and_family():
    # link.rs:102-157, family.rs:93-139
    assert abs(O.L.orc_inv_link(O.BINARY, 0.0) - 0.5) < 1e-10
    for mu in (0.1, 0.3, 0.5, 0.7, 0.9):
        assert abs(O.L.orc_inv_link(O.SURVIVAL, O.L.orc_link(O.SURVIVAL, mu)) - mu) < 1e-10
    assert abs(O.L.orc_update_mu(O.SURVIVAL, 0.0) - 0.6321205588) < 1e-6
    assert abs(O.L.orc_working_weight(O.BINARY, 0.5) - 0.25) < 1e-10
    assert O.L.orc_working_weight(O.QUANTITATIVE, 3.0) == 1.0


def test_irls_quantitative_known_answer():
    # ai_reml.rs:489-508: y = 1 + 2x exactly
    n = 100
    xi = np.arange(n) / n
    x = np.column_stack([np.ones(n), xi])
    a = O.fit_glm_irls(1 + 2 * xi, x, O.QUANTITATIVE)
    assert abs(a[0] - 1) < 0.1 and abs(a[1] - 2) < 0.1


def test_ai_reml_identity_grm_ranges():
    # ai_reml.rs:541-591 (identity GRM, quantitative, ranges only)
    n = 20
    y = 1.0 + 0.1 * np.arange(n)
    x = np.ones((n, 1))
    r = O.fit_ai_reml(y, x, O.QUANTITATIVE, O.K_IDENTITY, None, max_iter=10, tol=1e-4,
                      pcg_tol=1e-4, pcg_max_iter=100, n_random_vectors=5, seed=42)
    assert r["tau"][0] > 0 and r["tau"][1] >= 0
    assert 0 < r["iterations"] <= 10
    assert np.isfinite(r["log_likelihood"]) and r["log_likelihood"] < 0


@pytest.mark.parametrize("seed", range(0, 300, 15))
def test_otf_grm_matches_explicit(seed):
    # property_tests.rs:461-506: OnTheFlyGrm (f32) vs explicit GRM (f64) to 1e-5
    rng = np.random.default_rng(seed)
    n, m = 8, 15
    afs = 0.1 + rng.random(m) * 0.4
    r = rng.random((m, n))
    p0 = (1 - afs[:, None]) ** 2
    p1 = p0 + 2 * afs[:, None] * (1 - afs[:, None])
    dos = np.where(r < p0, 0.0, np.where(r < p1, 1.0, 2.0))
    v = rng.random(n) * 2 - 1
    k = O.grm_explicit(O.standardize(dos, afs, 0))
    otf = O.grm_matvec(O.standardize(dos, afs, 1), v, 1)
    assert np.abs(k @ v - otf).max() < 1e-5


def test_standardize_missing_is_exact_zero():
    dos = np.array([[0.0, np.nan, 2.0, 1.0]])
    z = O.standardize(dos, [0.3], 1)
    assert z[0, 1] == 0.0
    z0 = O.standardize(dos, [0.0], 0)  # denominator 0 -> zero column
    assert np.all(z0 == 0.0)


def test_packed_f64_product_equals_dense_fp64_product():
    spec = O.cohort_spec(n=701, m=300, seed=9, missing_rate=0.03)
    bed = O.gen_bed(spec)
    af, mac, nv = O.marker_stats(bed, 701, 300)
    keep = np.nonzero((af > 0.01) & (af < 0.99))[0]
    z = O.standardize(O.dosages(bed, 701, keep), af[keep], 0)
    v = np.random.default_rng(4).standard_normal((3, 701))
    got = O.grm_matmul_f64_packed(bed, 701, keep, af[keep], v)
    for c in range(3):
        want = O.grm_matvec(z, v[c], 0)
        assert np.abs(got[c] - want).max() <= 1e-12 * np.abs(want).max()
