"""The missing-call lists of the one-column products, on the CPU.

`mixed_model.kv_lists` lays the missing calls out as the GPU builder does (per thread
block and chunk, packed row/position entries; csrc/miss_lists.cu) and sums them as the
kernels do (contiguous per-thread slices, one add per run of equal rows; add_slice in
csrc/kernels_tc.cu). It must give the dense missing-flag model's product to the bit:
the missing sums are the same integers either way. The GPU kernels are held to the same
model in tests/test_gpu_mixed.py."""
import numpy as np
import pytest

import mixed_model as MM


def _codes(m, n, miss, seed):
    rng = np.random.default_rng(seed)
    af = rng.uniform(0.05, 0.5, m)
    # genotype codes 00 (2 copies), 10 (1), 11 (0) from HWE, then missing calls (01)
    g = rng.binomial(2, af[:, None], size=(m, n))
    codes = np.choose(g, [3, 2, 0]).astype(np.int64)
    codes[rng.random((m, n)) < miss] = 1
    return codes, af


@pytest.mark.parametrize("m,n,miss", [(300, 17000, 0.02),   # two pass-A sample chunks
                                      (2100, 600, 0.02),    # two pass-B marker chunks
                                      (130, 700, 0.0),      # no missing call at all
                                      (200, 900, 0.30)])    # long runs of one row
def test_list_sums_equal_dense_flag_sums(m, n, miss):
    codes, af = _codes(m, n, miss, seed=m + n)
    v = np.random.default_rng(1).standard_normal((n, 1))
    assert np.array_equal(MM.kv_lists(codes, af, v), MM.kv(codes, af, v))


def test_segments_cover_every_missing_call_once():
    codes, _ = _codes(200, 1100, 0.05, seed=3)
    m_pad, n_pad = 256, 1536
    miss = np.zeros((m_pad, n_pad), dtype=np.int8)
    miss[:200, :1100] = codes == 1
    total = int(miss.sum())
    off_a, ent_a, _ = MM.miss_segments_a(miss)
    off_b, ent_b, _ = MM.miss_segments_b(miss)
    assert off_a[-1] == off_b[-1] == total == len(ent_a) == len(ent_b)
    # within each segment the packed entries ascend (row, then position)
    for off, ent in ((off_a, ent_a), (off_b, ent_b)):
        for s in range(len(off) - 1):
            seg = ent[off[s]:off[s + 1]].astype(np.int64)
            assert np.all(np.diff(seg) > 0)
