"""saige_grm_matvec_dev_noalloc: the GRM product for callers that cannot allocate.

Some callers cannot let a library call cudaMalloc: a process whose own memory
pool already holds nearly all of the GPU's memory, or a latency-critical caller
that cannot afford the device synchronisation cudaMalloc/cudaFree may cause.
For them the library exports a variant of the FP32 product whose scratch is a
fixed array compiled into the library.  These tests call it through the C ABI
(ctypes, device pointers from torch tensors allocated before the calls) and hold
it to the existing entry point, saige_grm_matvec_dev, and to the FP64 oracle at
the FP32 product tolerance used throughout the GPU tests (2e-5 relative), on two
calls in a row with different vectors, so that a call that reused the previous
call's scratch contents would be caught.  The file is named to be collected last and works
both on its own in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import csaige_b200 as cs
from csaige_b200._lib import EINVAL, LIB, check
import oracle_ffi as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _grm(n, m, seed):
    spec = cs.CohortSpec(n=n, m=m, seed=seed, missing_rate=0.02)
    bed = cs.gen_bed(spec)
    af, _, _ = O.marker_stats(bed, n, m)
    keep = np.nonzero((af >= 0.01) & (af <= 0.99))[0]
    grm = cs.OnTheFlyGrm.from_bed(bed, n, m, keep, af[keep])
    return grm, bed, keep, af[keep]


def _scratch_bytes(grm):
    need, limit = C.c_size_t(), C.c_size_t()
    check(LIB.saige_grm_noalloc_scratch_bytes(grm._h, C.byref(need), C.byref(limit)))
    return need.value, limit.value


def _noalloc(grm, v, out, nrhs):
    return LIB.saige_grm_matvec_dev_noalloc(grm._h, C.c_void_p(v.data_ptr()),
                                            C.c_void_p(out.data_ptr()), grm.n_samples, nrhs,
                                            None)


@pytest.mark.parametrize("n,m,seed", [(1001, 300, 7), (20000, 3000, 5)])
def test_noalloc_matches_matvec_dev_on_two_calls(n, m, seed):
    grm, bed, keep, afs = _grm(n, m, seed)
    g = torch.Generator(device="cpu").manual_seed(seed)
    v1 = torch.randn(2, n, dtype=torch.float64, generator=g).cuda()  # two columns
    v2 = torch.randn(1, n, dtype=torch.float64, generator=g).cuda()
    want1 = torch.empty_like(v1)
    want2 = torch.empty_like(v2)
    got1 = torch.full_like(v1, float("nan"))
    got2 = torch.full_like(v2, float("nan"))
    grm.mat_vec_dev(v1.data_ptr(), want1.data_ptr(), nrhs=2, precision=cs.PREC_FP32)
    grm.mat_vec_dev(v2.data_ptr(), want2.data_ptr(), nrhs=1, precision=cs.PREC_FP32)
    torch.cuda.synchronize()

    check(_noalloc(grm, v1, got1, 2))
    torch.cuda.synchronize()
    free_after_first, _ = torch.cuda.mem_get_info()
    check(_noalloc(grm, v2, got2, 1))
    torch.cuda.synchronize()
    free_after_second, _ = torch.cuda.mem_get_info()

    w1, w2 = want1.cpu().numpy(), want2.cpu().numpy()
    r1, r2 = got1.cpu().numpy(), got2.cpu().numpy()
    assert np.isfinite(r1).all() and np.isfinite(r2).all()
    for c in range(2):
        assert _rel(r1[c], w1[c]) < 2e-5
    assert _rel(r2[0], w2[0]) < 2e-5
    # The second call found its scratch set up and allocated nothing.
    assert free_after_second == free_after_first
    # ... and both calls equal the FP64 oracle's product to the FP32 tolerance
    z = O.standardize(O.dosages(bed, n, keep), afs, 0)
    v1h, v2h = v1.cpu().numpy(), v2.cpu().numpy()
    for c in range(2):
        assert _rel(r1[c], O.grm_matvec(z, v1h[c], 0)) < 2e-5
    assert _rel(r2[0], O.grm_matvec(z, v2h[0], 0)) < 2e-5
    need, limit = _scratch_bytes(grm)
    assert 0 < need <= limit == 32 << 20


def test_noalloc_rejects_grm_beyond_static_scratch():
    # 3 million samples need about 36 MB of scratch (f32 v plus two partial-sum
    # planes), above the 32 MiB the library carries.
    n, m = 3_000_000, 256
    spec = cs.CohortSpec(n=n, m=m, seed=1)
    bed = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, bed.data_ptr())
    torch.cuda.synchronize()
    grm = cs.OnTheFlyGrm.from_bed_dev(bed.data_ptr(), spec.bed_len, n, m, np.arange(m),
                                      np.full(m, 0.3))
    del bed
    v = torch.zeros(1, n, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(v)
    need, limit = _scratch_bytes(grm)
    assert need > limit
    rc = _noalloc(grm, v, out, 1)
    assert rc == EINVAL
    msg = LIB.saige_last_error().decode()
    assert "static maximum" in msg
    # The existing entry point still serves this GRM.
    grm.mat_vec_dev(v.data_ptr(), out.data_ptr(), nrhs=1, precision=cs.PREC_FP32)
    torch.cuda.synchronize()
    grm.close()
