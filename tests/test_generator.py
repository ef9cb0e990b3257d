"""The oracle's statement of the seeded cohort generator equals the library's, byte
for byte (the CPU arm of the benchmark builds its cohorts with the oracle alone)."""
import numpy as np
import pytest

import csaige_b200 as cs
import oracle_ffi as O


@pytest.mark.parametrize("kw", [
    dict(),  # the plain fit-null cohort (N = 2,000, M = 5,000)
    dict(seed=7, n=3001, m=129, cousin_frac=0.02, missing_rate=0.05),
    dict(seed=12345, n=999, m=70, sib_frac=0.1, cousin_frac=0.02, trait=1, n_covar=4, h2=0.3),
    dict(seed=3, n=17, m=3, sib_frac=0.5, missing_rate=0.0, n_covar=0),
])
def test_oracle_generator_equals_library(kw):
    spec = cs.CohortSpec(**kw)
    ospec = O.cohort_spec(**kw)
    assert np.array_equal(O.gen_bed(ospec), cs.gen_bed(spec))
    y, x = cs.gen_pheno(spec)
    oy, ox = O.gen_pheno(ospec)
    assert np.array_equal(oy, y) and np.array_equal(ox, x)


def test_parallel_f32_product_is_the_reference_arithmetic():
    """kmode 2 (all threads, rayon-style chunks) against the one-thread f32 product:
    both are f32 sums of the same terms, so they agree to f32 rounding."""
    spec = O.cohort_spec(n=600, m=400, seed=5)
    bed = O.gen_bed(spec)
    af, mac, nv = O.marker_stats(bed, 600, 400)
    keep = np.nonzero((af > 0.01) & (af < 0.99))[0]
    z = O.standardize(O.dosages(bed, 600, keep), af[keep], 1)
    y, x = O.gen_pheno(spec)
    w = np.full(600, 0.2)
    b = np.random.default_rng(0).standard_normal(600)
    x1, it1, _, c1 = O.pcg_sigma(O.K_OTF, z, 600, z.shape[0], 1, w, [1.0, 0.3], b)
    x2, it2, _, c2 = O.pcg_sigma(O.K_OTF, z, 600, z.shape[0], 2, w, [1.0, 0.3], b)
    assert c1 and c2 and abs(it1 - it2) <= 1
    assert np.abs(x1 - x2).max() <= 1e-5 * np.abs(x1).max()
