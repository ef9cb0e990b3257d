"""CPU model of the MIXED-precision GRM product arithmetic (test infrastructure).

It restates, with numpy integers, exactly what the tensor-core path computes:
per-column 24-bit quantisation q = rint(x / (amax / (127*2^16))), exact integer
products of q with genotypes 0/1/2 and the missing indicator, and the same
FP64 rounding sequence in the epilogues.  The GPU output must equal it bit for
bit; the quantisation itself is judged separately against the FP64 oracle.
"""
import numpy as np

Q = 127.0 * 65536.0
LUT_G = np.array([2, 0, 1, 0], dtype=np.int64)


def codes(bed: np.ndarray, n_fam: int, markers, sample_idx=None) -> np.ndarray:
    bpm = (n_fam + 3) // 4
    sidx = np.arange(n_fam) if sample_idx is None else np.asarray(sample_idx)
    rows = bed[3:].reshape(-1, bpm)[np.asarray(markers)]
    return ((rows[:, sidx // 4] >> (2 * (sidx % 4)).astype(np.uint8)) & 3).astype(np.int64)


def meta(af):
    af = np.asarray(af, dtype=np.float64)
    denom = np.sqrt(2.0 * af * (1.0 - af))
    ok = denom > 1e-10
    inv_s = np.where(ok, 1.0 / np.where(ok, denom, 1.0), 0.0)
    two_p = np.where(ok, 2.0 * af, 0.0)
    return two_p, inv_s


def quantize(x: np.ndarray):
    amax = np.abs(x).max(axis=0)
    sc = np.where(amax > 0, amax / Q, 1.0)
    return np.rint(x / sc).astype(np.int64), sc


def kv(code_mat: np.ndarray, af, v: np.ndarray) -> np.ndarray:
    """K v for v of shape (n, R) with the MIXED arithmetic."""
    g = LUT_G[code_mat]
    miss = (code_mat == 1).astype(np.int64)
    two_p, inv_s = meta(af)
    m = code_mat.shape[0]
    qv, sv = quantize(v)
    G = g @ qv
    Mi = miss @ qv
    S = qv.sum(axis=0)
    t = G.astype(np.float64) - two_p[:, None] * (S[None, :] - Mi).astype(np.float64)
    u = inv_s[:, None] * (sv[None, :] * t)
    w = u * inv_s[:, None]
    c = w * two_p[:, None]
    qw, sw = quantize(w)
    qc, scc = quantize(c)
    Gw = g.T @ qw
    Mc = miss.T @ qc
    Sc = qc.sum(axis=0)
    out_scale = 1.0 / m
    return out_scale * ((sw[None, :] * Gw.astype(np.float64))
                        - (scc[None, :] * (Sc[None, :] - Mc).astype(np.float64)))
