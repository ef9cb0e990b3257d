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


# ---- missing-call lists (csrc/miss_lists.cu) ----------------------------------------
# The layout the one-column kernels consume: pass A segments = (block of A_ROWS marker
# rows, chunk of A_CHUNK samples), entries (row in block) << A_BITS | (sample in chunk),
# ordered by row then sample; pass B segments = (block of B_ROWS samples, chunk of B_CHUNK
# markers), entries (sample in block) << B_BITS | (marker in chunk), ordered by sample then
# marker.
A_ROWS, A_CHUNK, A_BITS = 64, 16384, 14
B_ROWS, B_CHUNK, B_BITS = 256, 2048, 11


def miss_segments_a(miss: np.ndarray):
    """miss: (m_pad, n_pad) 0/1. Returns (seg offsets, packed entries) of pass A."""
    m_pad, n_pad = miss.shape
    nch = -(-n_pad // A_CHUNK)
    ent, off = [], [0]
    for b in range(m_pad // A_ROWS):
        for c in range(nch):
            blk = miss[b * A_ROWS:(b + 1) * A_ROWS, c * A_CHUNK:(c + 1) * A_CHUNK]
            rows, pos = np.nonzero(blk)  # row-major: by row, then sample
            ent.append((rows.astype(np.uint64) << A_BITS) | pos.astype(np.uint64))
            off.append(off[-1] + len(rows))
    return np.array(off, dtype=np.int64), np.concatenate(ent).astype(np.uint32), nch


def miss_segments_b(miss: np.ndarray):
    """Pass B segments of the same calls, from the samples' side."""
    m_pad, n_pad = miss.shape
    nch = -(-m_pad // B_CHUNK)
    ent, off = [], [0]
    for p in range(n_pad // B_ROWS):
        for c in range(nch):
            blk = miss[c * B_CHUNK:(c + 1) * B_CHUNK, p * B_ROWS:(p + 1) * B_ROWS].T
            smp, pos = np.nonzero(blk)  # by sample, then marker
            ent.append((smp.astype(np.uint64) << B_BITS) | pos.astype(np.uint64))
            off.append(off[-1] + len(smp))
    return np.array(off, dtype=np.int64), np.concatenate(ent).astype(np.uint32), nch


def slice_sums(ent, e0, e1, nt, bits, n_tags, value):
    """The kernels' add_slice over one segment: nt threads take contiguous slices of
    ceil(len / nt) entries and add value(position) per run of equal tags (exact int)."""
    out = np.zeros(n_tags, dtype=np.int64)
    ln = -(-(e1 - e0) // nt) if e1 > e0 else 0
    mask = (1 << bits) - 1
    for t in range(nt):
        lo = e0 + t * ln
        hi = min(lo + ln, e1)
        if lo >= hi:
            continue
        x = ent[lo:hi].astype(np.int64)
        tags, vals = x >> bits, value(x & mask)
        for tag in np.unique(tags):  # each run adds once; equal tags are contiguous
            out[tag] += int(vals[tags == tag].sum())
    return out


def kv_lists(code_mat: np.ndarray, af, v: np.ndarray) -> np.ndarray:
    """kv() for one column with Mi and Mc summed over the segment lists (pass A: 256
    threads per block, pass B: 128), padded to the kernels' m_pad / n_pad."""
    assert v.shape[1] == 1
    m, n = code_mat.shape
    m_pad, n_pad = -(-m // 128) * 128, -(-n // 512) * 512
    miss = np.zeros((m_pad, n_pad), dtype=np.int8)
    miss[:m, :n] = code_mat == 1
    g = LUT_G[code_mat]
    two_p, inv_s = meta(af)
    qv, sv = quantize(v)
    q_pad = np.zeros(n_pad, dtype=np.int64)
    q_pad[:n] = qv[:, 0]
    off, ent, nch = miss_segments_a(miss)
    Mi = np.zeros(m_pad, dtype=np.int64)
    for b in range(m_pad // A_ROWS):
        for c in range(nch):
            s = b * nch + c
            Mi[b * A_ROWS:(b + 1) * A_ROWS] += slice_sums(
                ent, off[s], off[s + 1], 256, A_BITS, A_ROWS,
                lambda pos, c=c: q_pad[c * A_CHUNK + pos])
    G = g @ qv
    S = qv.sum(axis=0)
    t = G.astype(np.float64) - two_p[:, None] * (S[None, :] - Mi[:m, None]).astype(np.float64)
    u = inv_s[:, None] * (sv[None, :] * t)
    w = u * inv_s[:, None]
    c_ = w * two_p[:, None]
    qw, sw = quantize(w)
    qc, scc = quantize(c_)
    qc_pad = np.zeros(m_pad, dtype=np.int64)
    qc_pad[:m] = qc[:, 0]
    off, ent, nch = miss_segments_b(miss)
    Mc = np.zeros(n_pad, dtype=np.int64)
    for p in range(n_pad // B_ROWS):
        for c in range(nch):
            s = p * nch + c
            Mc[p * B_ROWS:(p + 1) * B_ROWS] += slice_sums(
                ent, off[s], off[s + 1], 128, B_BITS, B_ROWS,
                lambda pos, c=c: qc_pad[c * B_CHUNK + pos])
    Gw = g.T @ qw
    Sc = qc.sum(axis=0)
    return (1.0 / m) * ((sw[None, :] * Gw.astype(np.float64))
                        - (scc[None, :] * (Sc[None, :] - Mc[:n, None]).astype(np.float64)))
