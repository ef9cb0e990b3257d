"""Explicit GRM on the GPU (compute_dense_grm, compute_sparse_grm and the dosage forms,
saige-core/src/grm/dense.rs:22-186, grm/sparse.rs:18-98) through the C ABI, against
the CPU oracle's restatement.

With GRM_ARITH_REFERENCE every entry is one f64 sum in marker order with a rounded
multiply and a rounded add, as the reference forms it, so the GPU matrix must equal
the oracle's bit for bit; the sparse form must list exactly the oracle's entries."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O

pytestmark = pytest.mark.gpu


def _cohort(n, m, seed, missing=0.01, sib=0.2, maf_lo=0.005):
    spec = cs.CohortSpec(n=n, m=m, seed=seed, missing_rate=missing, sib_frac=sib,
                         cousin_frac=0.1, maf_lo=maf_lo, maf_hi=0.5)
    return cs.gen_bed(spec)


@pytest.fixture(scope="module")
def bed1000():
    return _cohort(1000, 700, 11)


@pytest.mark.parametrize("n,m,seed", [(1000, 700, 11), (333, 250, 3), (129, 64, 5), (7, 40, 9),
                                      (1, 5, 2)])
def test_dense_is_bit_identical_to_oracle(n, m, seed):
    bed = _cohort(n, m, seed)
    k, used = cs.compute_dense_grm(bed, n, m)
    want, used_o = O.dense_grm_bed(bed, n, m)
    assert used == used_o
    assert np.array_equal(k, want)


def test_sample_subset_and_maf_window(bed1000):
    rng = np.random.default_rng(0)
    sidx = rng.permutation(1000)[:517]
    for min_maf in (0.0, 0.05, 0.3):
        k, used = cs.compute_dense_grm(bed1000, 1000, 700, min_maf=min_maf, sample_idx=sidx)
        want, used_o = O.dense_grm_bed(bed1000, 1000, 700, min_maf=min_maf, sample_idx=sidx)
        assert used == used_o and np.array_equal(k, want), min_maf


def test_no_marker_used_gives_zeros(bed1000):
    k, used = cs.compute_dense_grm(bed1000, 1000, 700, min_maf=0.6)
    assert used == 0 and k.shape == (1000, 1000) and not k.any()
    g, used = cs.compute_sparse_grm(bed1000, 1000, 700, min_maf=0.6)
    assert used == 0 and g.vals.size == 1000 and np.array_equal(g.rows, g.cols)
    assert not g.vals.any()


@pytest.mark.parametrize("cutoff", [0.125, 0.02, -1.0])
def test_sparse_lists_the_oracle_entries(bed1000, cutoff):
    # cutoff -1 keeps every entry of the upper triangle: more than the first capacity guess
    g, used = cs.compute_sparse_grm(bed1000, 1000, 700, relatedness_cutoff=cutoff)
    k, used_o = O.dense_grm_bed(bed1000, 1000, 700)
    r, c, v = O.sparse_from_dense(k, cutoff)
    assert used == used_o == g.n_markers_used and g.n == 1000
    assert np.array_equal(g.rows, r) and np.array_equal(g.cols, c) and np.array_equal(g.vals, v)
    if cutoff == 0.125:
        assert g.vals.size > 1000  # the cohort has related pairs


def test_fma_arithmetic_is_close(bed1000):
    k, _ = cs.compute_dense_grm(bed1000, 1000, 700, arith=cs.GRM_ARITH_FMA)
    want, _ = O.dense_grm_bed(bed1000, 1000, 700)
    assert np.allclose(k, want, rtol=1e-12, atol=1e-14)


def test_dosage_form_is_bit_identical_to_oracle():
    rng = np.random.default_rng(7)
    m, n = 90, 300
    af = rng.uniform(0.0, 0.5, m)
    af[3] = 0.0                                     # 2 af (1 - af) < 1e-10: skipped
    d = rng.binomial(2, af[:, None], (m, n)).astype(float)
    d[:, :5] += rng.uniform(-0.3, 0.3, (m, 5))      # non-integer dosages
    d[rng.random((m, n)) < 0.03] = np.nan
    for arith in (cs.GRM_ARITH_REFERENCE,):
        k = cs.compute_grm_from_dosages(d, af, arith=arith)
        want, used = O.grm_from_dosages(d, af)
        assert used == m - 1 and np.array_equal(k, want)
    g = cs.compute_sparse_grm_from_dosages(d, af, 0.05)
    r, c, v = O.sparse_from_dense(want, 0.05)
    assert np.array_equal(g.rows, r) and np.array_equal(g.cols, c) and np.array_equal(g.vals, v)
    assert cs.compute_grm_from_dosages(np.zeros((0, 4)), []).shape == (0, 0)


def test_reference_unit_cases_on_the_gpu():
    # dense.rs:231-251 and sparse.rs:105-118 inputs
    d = np.array([[0, 1, 2, 1], [2, 1, 0, 1], [1, 1, 1, 1.0]])
    k = cs.compute_grm_from_dosages(d, [0.5, 0.5, 0.5])
    assert np.array_equal(k, O.grm_from_dosages(d, [0.5] * 3)[0]) and np.array_equal(k, k.T)
    g = cs.compute_sparse_grm_from_dosages(np.array([[0, 2, 0, 2.0]] * 3), [0.5] * 3, 0.5)
    assert 4 <= g.nnz <= 16


@pytest.mark.parametrize("n,m", [(2048, 1500), (1000, 700)])
def test_dense_agrees_with_the_on_the_fly_product(n, m):
    # two independent GPU paths and the oracle's FP64 on-the-fly product (pcg.rs:128-180)
    bed = _cohort(n, m, 21, missing=0.0)
    k, used = cs.compute_dense_grm(bed, n, m, min_maf=0.0)
    af, _, _ = cs.bed_marker_stats(bed, n, m)
    idx = np.nonzero(2.0 * af * (1.0 - af) >= 1e-10)[0]
    assert idx.size == used
    v = np.random.default_rng(1).standard_normal((3, n))
    z = O.standardize(O.dosages(bed, n, idx), af[idx], 0)
    want = np.stack([O.grm_matvec(z, v[j], 0) for j in range(3)])
    err_dense = np.max(np.abs(v @ k - want))
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, idx, af[idx], precision=cs.PREC_MIXED)
    err_otf = np.max(np.abs(grm.mat_vec(v) - want))
    assert err_dense < 1e-9 * np.max(np.abs(want)), (err_dense, err_otf)
    assert err_otf < 1e-6 * np.max(np.abs(want)), (err_dense, err_otf)


def test_create_sparse_grm_files(tmp_path):
    n, m = 400, 300
    bed = _cohort(n, m, 13)
    pre = tmp_path / "geno"
    (tmp_path / "geno.bed").write_bytes(bytes(bed))
    (tmp_path / "geno.fam").write_text("".join(f"F{i} I{i} 0 0 1 -9\n" for i in range(n)))
    (tmp_path / "geno.bim").write_text("".join(f"1 rs{j} 0 {j + 1} A G\n" for j in range(m)))
    g, used, mtx, ids = cs.create_sparse_grm(pre, tmp_path / "res")
    k, used_o = O.dense_grm_bed(bed, n, m)
    r, c, v = O.sparse_from_dense(k, 0.125)
    assert used == used_o
    assert open(mtx).read() == O.sparse_grm_text(n, r, c, v)
    assert open(ids).read() == "".join(f"I{i}\n" for i in range(n))
    assert mtx.endswith("res.sparseGRM.mtx") and ids.endswith("res.sparseGRM.mtx.sampleIDs.txt")
