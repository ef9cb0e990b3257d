"""The bounded waits of the tensor-core product (csrc/kernels_tc.cu).

A wait budget of 0 makes every pipeline wait that is not already satisfied give up at
once, so the product takes its abort path: no further copy or MMA is issued, the
copies and MMAs already issued are waited for, the tensor memory is freed and the call
reports SAIGE_TIMEOUT.  The next product on the same handle, with the default budget,
must then be exact (bit-identical to the CPU model of the arithmetic)."""
import numpy as np
import pytest

import csaige_b200 as cs
import mixed_model as MM
import oracle_ffi as O
from csaige_b200 import _lib

pytestmark = pytest.mark.gpu


def test_timed_out_product_reports_timeout_and_handle_stays_usable():
    n, m = 4096, 2048
    spec = cs.CohortSpec(n=n, m=m, seed=17, missing_rate=0.02)
    bed = cs.gen_bed(spec)
    af, mac, nv = O.marker_stats(bed, n, m)
    keep = np.nonzero((af >= 0.01) & (af <= 0.99))[0]
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, keep, af[keep], precision=cs.PREC_MIXED)
    v = np.random.default_rng(5).standard_normal((5, n))
    want = MM.kv(MM.codes(bed, n, keep), af[keep], v.T).T
    assert np.array_equal(grm.mat_vec(v), want)
    try:
        _lib.LIB.saige_tc_set_wait_budget(0)
        with pytest.raises(cs.SaigeError) as e:
            grm.mat_vec(v)
        assert e.value.code == _lib.TIMEOUT
    finally:
        _lib.LIB.saige_tc_set_wait_budget(-1)
    for _ in range(2):
        assert np.array_equal(grm.mat_vec(v), want)
