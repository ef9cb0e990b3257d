"""Explicit GRM (saige-core/src/grm/dense.rs, grm/sparse.rs, saige-geno/src/
sparse_grm_io.rs): the oracle pinned against the reference's own GRM tests, and the
library's host-side pieces (writer, reader, PLINK text files, argument checks) on
the CPU."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O


def _chacha_cohort(seed: int, n: int, m: int):
    """The generator of dense.rs:193-215 and property_tests.rs:470-485: ChaCha8 from
    seed_from_u64, af = 0.1 + 0.4 u, genotype thresholds (1-af)^2 and + 2 af (1-af)."""
    rng = O.chacha8(seed)
    dos, afs = [], []
    for _ in range(m):
        af = 0.1 + O.gen_f64(rng) * 0.4
        g = []
        for _ in range(n):
            r = O.gen_f64(rng)
            q = (1.0 - af) * (1.0 - af)
            g.append(0.0 if r < q else (1.0 if r < q + 2.0 * af * (1.0 - af) else 2.0))
        dos.append(g)
        afs.append(af)
    return np.array(dos), np.array(afs), rng


def test_oracle_symmetric_case():
    # dense.rs:231-251 (test_grm_symmetric): symmetric; the constant marker is still used
    d = np.array([[0, 1, 2, 1], [2, 1, 0, 1], [1, 1, 1, 1.0]])
    k, used = O.grm_from_dosages(d, [0.5, 0.5, 0.5])
    assert used == 3
    assert np.array_equal(k, k.T)
    z = (0.0 - 1.0) / np.sqrt(0.5)
    assert k[0, 0] == (z * z + z * z + 0.0 * 0.0) * (1.0 / 3)
    assert k[0, 2] == (z * -z + -z * z + 0.0 * 0.0) * (1.0 / 3)


def test_oracle_identity_like_case():
    # dense.rs:193-228 (test_grm_identity_like): ChaCha8 seed 42, n 5, m 500, diagonal > 0
    d, afs, _ = _chacha_cohort(42, 5, 500)
    k, used = O.grm_from_dosages(d, afs)
    assert used == 500 and k.shape == (5, 5)
    assert np.all(np.diag(k) > 0)


def test_oracle_sparse_cutoff_case():
    # sparse.rs:105-118 (test_sparse_grm_cutoff)
    d = np.array([[0, 2, 0, 2.0]] * 3)
    k, _ = O.grm_from_dosages(d, [0.5] * 3)
    r, c, v = O.sparse_from_dense(k, 0.5)
    nnz = 2 * v.size - np.count_nonzero(r == c)
    assert 4 <= nnz <= 16


@pytest.mark.parametrize("seed", [0, 1, 7, 123, 299])
def test_oracle_explicit_matches_on_the_fly(seed):
    # property_tests.rs:461-506: explicit K v against the f32 on-the-fly product, < 1e-5
    d, afs, rng = _chacha_cohort(seed, 8, 15)
    k, _ = O.grm_from_dosages(d, afs)
    v = np.array([O.gen_f64(rng) * 2.0 - 1.0 for _ in range(8)])
    z32 = O.standardize(d, afs, 1)
    otf = O.grm_matvec(z32, v, 1)
    assert np.max(np.abs(k @ v - otf)) < 1e-5


def test_oracle_bed_equals_dosage_form():
    # dense.rs:22-112 on a .bed is dense.rs:115-186 on its dosages after the af window
    spec = cs.CohortSpec(n=150, m=90, seed=4, missing_rate=0.02, maf_lo=0.001, maf_hi=0.5)
    bed = cs.gen_bed(spec)
    k, used = O.dense_grm_bed(bed, 150, 90, min_maf=0.05)
    af, _, _ = O.marker_stats(bed, 150, 90)
    keep = np.nonzero((af >= 0.05) & (af <= 0.95))[0]
    k2, used2 = O.grm_from_dosages(O.dosages(bed, 150, keep), af[keep])
    assert used == used2 == keep.size and np.array_equal(k, k2)


def test_oracle_no_marker_gives_zeros():
    spec = cs.CohortSpec(n=40, m=10, seed=1)
    bed = cs.gen_bed(spec)
    k, used = O.dense_grm_bed(bed, 40, 10, min_maf=0.6)  # af < 0.6 or af > 0.4: every marker
    assert used == 0 and not k.any()
    assert O.grm_from_dosages(np.zeros((0, 4)), [])[0].shape == (0, 0)


# ---- host pieces of the library (no GPU needed) ------------------------------------
def test_read_sparse_grm_reference_case(tmp_path):
    # sparse_grm_io.rs:118-150 (test_read_write_sparse_grm)
    mtx, ids = tmp_path / "test.sparseGRM.mtx", tmp_path / "test.sparseGRM.mtx.sampleIDs.txt"
    mtx.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 4\n1 1 1.0\n2 2 1.0\n"
                   "3 3 1.0\n1 2 0.25\n")
    ids.write_text("S1\nS2\nS3\n")
    g, names = cs.read_sparse_grm(mtx, ids)
    assert names == ["S1", "S2", "S3"] and g.n == 3
    assert abs(g.get(0, 0) - 1.0) < 1e-10
    assert abs(g.get(0, 1) - 0.25) < 1e-10 and abs(g.get(1, 0) - 0.25) < 1e-10
    assert g.nnz == 5 and g.get(0, 2) == 0.0


def test_writer_text_matches_restated_format(tmp_path):
    rng = np.random.default_rng(3)
    n = 30
    k = rng.normal(0, 0.1, (n, n))
    k = (k + k.T) / 2 + np.eye(n)
    k[2, 7] = k[7, 2] = -0.2   # negative entries pass on |K|
    k[1, 4] = k[4, 1] = 1e-13  # below the cutoff
    r, c, v = O.sparse_from_dense(k, 0.125)
    g = cs.SparseGrm(n, r, c, v)
    ids = [f"id{i}" for i in range(n)]
    cs.write_sparse_grm(g, ids, tmp_path / "a.mtx", tmp_path / "a.ids")
    assert (tmp_path / "a.mtx").read_text() == O.sparse_grm_text(n, r, c, v)
    assert (tmp_path / "a.ids").read_text() == "".join(s + "\n" for s in ids)
    back, names = cs.read_sparse_grm(tmp_path / "a.mtx", tmp_path / "a.ids")
    assert names == ids and np.array_equal(back.rows, r) and np.array_equal(back.cols, c)
    assert np.allclose(back.vals, v, rtol=0, atol=5e-11)


def test_writer_rejects_entries_off_the_upper_triangle(tmp_path):
    bad = cs.SparseGrm(3, np.array([1, 0], np.int32), np.array([0, 0], np.int32),
                       np.array([0.5, 1.0]))
    with pytest.raises(cs.SaigeError, match="upper triangle"):
        cs.write_sparse_grm(bad, ["a", "b", "c"], tmp_path / "b.mtx", tmp_path / "b.ids")
    unsorted = cs.SparseGrm(3, np.array([1, 0], np.int32), np.array([1, 0], np.int32),
                            np.array([1.0, 1.0]))
    with pytest.raises(cs.SaigeError, match="sorted"):
        cs.write_sparse_grm(unsorted, ["a", "b", "c"], tmp_path / "b.mtx", tmp_path / "b.ids")


def test_output_names_follow_with_extension():
    # create_sparse_grm.rs:53-55
    assert cs.api._with_extension("out/example", "sparseGRM.mtx") == "out/example.sparseGRM.mtx"
    assert (cs.api._with_extension("out/example", "sparseGRM.mtx.sampleIDs.txt")
            == "out/example.sparseGRM.mtx.sampleIDs.txt")


def _write_plink(prefix, bed, n, m, fam_fields=6):
    (prefix.parent / (prefix.name + ".bed")).write_bytes(bytes(bed))
    (prefix.parent / (prefix.name + ".fam")).write_text(
        "".join(" ".join([f"f{i}", f"s{i}", "0", "0", "1", "-9"][:fam_fields]) + "\n"
                for i in range(n)))
    (prefix.parent / (prefix.name + ".bim")).write_text(
        "".join(f"1\trs{j}\t0\t{100 + j}\tA\tG\n" for j in range(m)))


def test_read_plink_checks(tmp_path):
    spec = cs.CohortSpec(n=21, m=7, seed=2)
    bed = cs.gen_bed(spec)
    pre = tmp_path / "geno"
    _write_plink(pre, bed, 21, 7)
    p = cs.read_plink(pre)
    assert (p.n_fam, p.m_tot) == (21, 7) and p.sample_ids[3] == "s3" and p.marker_ids[6] == "rs6"
    assert np.array_equal(p.bed, bed)
    (tmp_path / "geno.bed").write_bytes(bytes(bed[:-1]))
    with pytest.raises(ValueError, match="too small"):
        cs.read_plink(pre)
    _write_plink(pre, bed, 21, 7, fam_fields=5)
    with pytest.raises(ValueError, match="fewer than 6 fields"):
        cs.read_plink(pre)


def test_config_defaults_are_the_command_defaults():
    import ctypes as C
    from csaige_b200 import _lib
    cfg = _lib.ExplicitGrmConfigC()
    assert _lib.LIB.saige_explicit_grm_config_default(C.byref(cfg)) == 0
    assert cfg.min_maf == 0.01 and cfg.relatedness_cutoff == 0.125
    assert cfg.arith == cs.GRM_ARITH_REFERENCE and cfg.device == -1
