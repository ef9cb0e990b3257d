"""Explicit GRM over the sm_100a library: the host mirror of

  compute_dense_grm                  saige-core/src/grm/dense.rs:22-112
  compute_grm_from_dosages           saige-core/src/grm/dense.rs:115-186
  compute_sparse_grm                 saige-core/src/grm/sparse.rs:18-66
  compute_sparse_grm_from_dosages    saige-core/src/grm/sparse.rs:69-98
  read_sparse_grm / write_sparse_grm saige-geno/src/sparse_grm_io.rs:16-115
  PlinkReader::new (.fam/.bim/.bed)  saige-geno/src/plink.rs:62-168
  create-sparse-grm                  saige-cli/src/commands/create_sparse_grm.rs:37-71

The GRM itself is computed by the library (one FP64 kernel; with
GRM_ARITH_REFERENCE every entry is bit-identical to the reference's); this module
only moves arrays, parses the PLINK text files and reads .mtx files back.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import LIB, SaigeError, check
from .api import _bed_array, _dptr, _f64, _i64ptr, _with_extension

GRM_ARITH_REFERENCE = 0  # rounded multiply, then rounded add, in marker order (the reference)
GRM_ARITH_FMA = 1        # fused multiply-add: twice the FP64 rate, last-bit differences


@dataclass
class ExplicitGrmInfo:
    n_markers_used: int
    nnz: int
    kernel_seconds: float
    total_seconds: float
    terms: float  # n (n + 1) / 2 * n_markers_used products summed


@dataclass
class SparseGrm:
    """A symmetric sparse GRM stored as its upper triangle with the diagonal, sorted by
    row then column: the entries write_sparse_grm lists (sparse_grm_io.rs:92-107)."""
    n: int
    rows: np.ndarray  # int32, 0-based
    cols: np.ndarray
    vals: np.ndarray
    n_markers_used: int = 0
    info: Optional[ExplicitGrmInfo] = field(default=None, repr=False)

    @property
    def nnz(self) -> int:
        """Stored entries of the full symmetric matrix (SparseMatrix::nnz)."""
        return int(2 * self.vals.size - np.count_nonzero(self.rows == self.cols))

    def get(self, i: int, j: int) -> float:
        a, b = (i, j) if i <= j else (j, i)
        lo = np.searchsorted(self.rows, a, side="left")
        hi = np.searchsorted(self.rows, a, side="right")
        k = lo + np.searchsorted(self.cols[lo:hi], b)
        return float(self.vals[k]) if k < hi and self.cols[k] == b else 0.0

    def to_dense(self) -> np.ndarray:
        k = np.zeros((self.n, self.n))
        k[self.rows, self.cols] = self.vals
        k[self.cols, self.rows] = self.vals
        return k


def _config(min_maf: float, cutoff: float, arith: int, device: int):
    cfg = _lib.ExplicitGrmConfigC()
    check(LIB.saige_explicit_grm_config_default(C.byref(cfg)))
    cfg.min_maf = float(min_maf)
    cfg.relatedness_cutoff = float(cutoff)
    cfg.arith = int(arith)
    cfg.device = int(device)
    return cfg


def _info(i) -> ExplicitGrmInfo:
    return ExplicitGrmInfo(int(i.n_markers_used), int(i.nnz), float(i.kernel_seconds),
                           float(i.total_seconds), float(i.terms))


def _take_sparse(handle: C.c_void_p, info) -> SparseGrm:
    try:
        n = int(LIB.saige_sparse_grm_n(handle))
        nnz = int(LIB.saige_sparse_grm_nnz(handle))
        rows = np.empty(nnz, np.int32)
        cols = np.empty(nnz, np.int32)
        vals = np.empty(nnz, np.float64)
        check(LIB.saige_sparse_grm_get(handle, rows.ctypes.data_as(C.POINTER(C.c_int32)),
                                       cols.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(vals)))
        used = int(LIB.saige_sparse_grm_n_markers(handle))
    finally:
        LIB.saige_sparse_grm_free(handle)
    return SparseGrm(n, rows, cols, vals, used, _info(info))


def _bed_args(bed, n_fam: int, sample_idx):
    b = _bed_array(bed)
    sidx = None if sample_idx is None else np.ascontiguousarray(sample_idx, dtype=np.int64)
    n = n_fam if sidx is None else sidx.size
    return b, sidx, n


def compute_dense_grm(bed, n_fam: int, m_tot: int, min_maf: float = 0.01,
                      sample_idx: Optional[Sequence[int]] = None,
                      arith: int = GRM_ARITH_REFERENCE, device: int = -1,
                      info_out: Optional[list] = None) -> tuple[np.ndarray, int]:
    """compute_dense_grm (dense.rs:22-112) on .bed bytes: (K n x n, markers used)."""
    b, sidx, n = _bed_args(bed, n_fam, sample_idx)
    out = np.empty((n, n))
    info = _lib.ExplicitGrmInfoC()
    check(LIB.saige_dense_grm_from_bed(b.ctypes.data_as(C.POINTER(C.c_uint8)), b.size, n_fam,
                                       m_tot, _i64ptr(sidx), n,
                                       C.byref(_config(min_maf, 0.0, arith, device)), _dptr(out),
                                       C.byref(info)))
    if info_out is not None:
        info_out.append(_info(info))
    return out, int(info.n_markers_used)


def compute_sparse_grm(bed, n_fam: int, m_tot: int, min_maf: float = 0.01,
                       relatedness_cutoff: float = 0.125,
                       sample_idx: Optional[Sequence[int]] = None,
                       arith: int = GRM_ARITH_REFERENCE, device: int = -1
                       ) -> tuple[SparseGrm, int]:
    """compute_sparse_grm (sparse.rs:18-66): (sparse K, markers used)."""
    b, sidx, n = _bed_args(bed, n_fam, sample_idx)
    h = C.c_void_p()
    info = _lib.ExplicitGrmInfoC()
    check(LIB.saige_sparse_grm_from_bed(b.ctypes.data_as(C.POINTER(C.c_uint8)), b.size, n_fam,
                                        m_tot, _i64ptr(sidx), n,
                                        C.byref(_config(min_maf, relatedness_cutoff, arith,
                                                        device)),
                                        C.byref(h), C.byref(info)))
    g = _take_sparse(h, info)
    return g, g.n_markers_used


def _dosage_args(dosages, allele_freqs):
    d = np.asarray(dosages, dtype=np.float64)
    if d.ndim != 2:
        raise SaigeError(_lib.EINVAL, "dosages must be a 2-D array (markers x samples)")
    d = np.ascontiguousarray(d)
    af = _f64(allele_freqs, d.shape[0])
    return d, af


def compute_grm_from_dosages(dosages, allele_freqs, arith: int = GRM_ARITH_REFERENCE,
                             device: int = -1) -> np.ndarray:
    """compute_grm_from_dosages (dense.rs:115-186): dosages markers x samples (NaN =
    missing); no marker rows give the 0 x 0 matrix."""
    d, af = _dosage_args(dosages, allele_freqs)
    m, n = d.shape
    if m == 0:
        return np.zeros((0, 0))
    out = np.empty((n, n))
    info = _lib.ExplicitGrmInfoC()
    check(LIB.saige_grm_from_dosages(_dptr(d), _dptr(af), n, m,
                                     C.byref(_config(0.0, 0.0, arith, device)), _dptr(out),
                                     C.byref(info)))
    return out


def compute_sparse_grm_from_dosages(dosages, allele_freqs, relatedness_cutoff: float,
                                    arith: int = GRM_ARITH_REFERENCE,
                                    device: int = -1) -> SparseGrm:
    """compute_sparse_grm_from_dosages (sparse.rs:69-98)."""
    d, af = _dosage_args(dosages, allele_freqs)
    m, n = d.shape
    h = C.c_void_p()
    info = _lib.ExplicitGrmInfoC()
    check(LIB.saige_sparse_grm_from_dosages(_dptr(d), _dptr(af), n, m,
                                            C.byref(_config(0.0, relatedness_cutoff, arith,
                                                            device)),
                                            C.byref(h), C.byref(info)))
    return _take_sparse(h, info)


def write_sparse_grm(matrix: SparseGrm, sample_ids: Sequence[str], mtx_path, ids_path) -> None:
    """write_sparse_grm (sparse_grm_io.rs:73-115), through the library's writer."""
    ids = [str(s).encode() for s in sample_ids]
    arr = (C.c_char_p * max(len(ids), 1))(*ids)
    rows = np.ascontiguousarray(matrix.rows, np.int32)
    cols = np.ascontiguousarray(matrix.cols, np.int32)
    vals = np.ascontiguousarray(matrix.vals, np.float64)
    h = C.c_void_p()
    check(LIB.saige_sparse_grm_from_triplets(matrix.n, vals.size,
                                             rows.ctypes.data_as(C.POINTER(C.c_int32)),
                                             cols.ctypes.data_as(C.POINTER(C.c_int32)),
                                             _dptr(vals), matrix.n_markers_used, C.byref(h)))
    try:
        check(LIB.saige_write_sparse_grm(h, arr, len(ids), str(mtx_path).encode(),
                                         str(ids_path).encode()))
    finally:
        LIB.saige_sparse_grm_free(h)


def read_sparse_grm(mtx_path, ids_path) -> tuple[SparseGrm, list]:
    """read_sparse_grm (sparse_grm_io.rs:16-69): sample IDs (trimmed, empty lines
    dropped), the first non-comment line as the dimensions, then 1-based "row col value"
    entries; an off-diagonal entry stands for both (r, c) and (c, r), and repeated
    entries add up (TriMat::to_csr)."""
    with open(ids_path) as f:
        ids = [ln.strip() for ln in f.read().splitlines() if ln.strip()]
    n = len(ids)
    acc: dict = {}
    header_done = False
    with open(mtx_path) as f:
        for line in f.read().splitlines():
            line = line.strip()
            if line.startswith("%") or line.startswith("#"):
                continue
            if not header_done:
                header_done = True
                continue
            fields = line.split()
            if len(fields) >= 3:
                r, c, v = int(fields[0]) - 1, int(fields[1]) - 1, float(fields[2])
                if r < 0 or c < 0:
                    raise ValueError(f"bad index in {mtx_path}: {line}")
                key = (r, c) if r <= c else (c, r)
                acc[key] = acc.get(key, 0.0) + v
    keys = sorted(acc)
    rows = np.array([k[0] for k in keys], dtype=np.int32)
    cols = np.array([k[1] for k in keys], dtype=np.int32)
    vals = np.array([acc[k] for k in keys], dtype=np.float64)
    return SparseGrm(n, rows, cols, vals), ids


@dataclass
class PlinkFiles:
    """A PLINK binary fileset as PlinkReader::new opens it (plink.rs:62-112)."""
    bed: np.ndarray       # the whole .bed, header included
    n_fam: int
    m_tot: int
    sample_ids: list      # IID column of the .fam
    chroms: list          # .bim column 1
    marker_ids: list      # .bim column 2


def _parse_table(path: str, what: str) -> list:
    rows = []
    with open(path) as f:
        for k, line in enumerate(f.read().splitlines()):
            line = line.strip()
            if not line:
                continue
            fields = line.split()
            if len(fields) < 6:
                raise ValueError(f"{what} file line {k + 1} has fewer than 6 fields")
            rows.append(fields)
    return rows


def read_plink(plink_file) -> PlinkFiles:
    """Open <prefix>.bed/.bim/.fam (Path::with_extension on the prefix) with the
    reference's checks: six fields per .fam/.bim line, the .bed magic, SNP-major mode
    and size."""
    fam = _parse_table(_with_extension(plink_file, "fam"), "Fam")
    bim = _parse_table(_with_extension(plink_file, "bim"), "Bim")
    bed = np.fromfile(_with_extension(plink_file, "bed"), dtype=np.uint8)
    n, m = len(fam), len(bim)
    if bed.size < 3:
        raise ValueError("Bed file too small")
    if bed[0] != 0x6C or bed[1] != 0x1B:
        raise ValueError("Invalid PLINK bed file magic number")
    if bed[2] != 0x01:
        raise ValueError("Only SNP-major bed files are supported (mode byte = 0x01)")
    want = 3 + (n + 3) // 4 * m
    if bed.size < want:
        raise ValueError(f"Bed file too small: expected at least {want} bytes, got {bed.size}")
    return PlinkFiles(bed, n, m, [r[1] for r in fam], [r[0] for r in bim], [r[1] for r in bim])


def create_sparse_grm(plink_file, output_prefix, relatedness_cutoff: float = 0.125,
                      min_maf: float = 0.01, arith: int = GRM_ARITH_REFERENCE,
                      device: int = -1) -> tuple:
    """The create-sparse-grm command (create_sparse_grm.rs:37-71): writes
    <prefix>.sparseGRM.mtx and <prefix>.sparseGRM.mtx.sampleIDs.txt; returns
    (sparse GRM, markers used, mtx path, IDs path)."""
    p = read_plink(plink_file)
    g, used = compute_sparse_grm(p.bed, p.n_fam, p.m_tot, min_maf, relatedness_cutoff,
                                 arith=arith, device=device)
    mtx = _with_extension(output_prefix, "sparseGRM.mtx")
    ids = _with_extension(output_prefix, "sparseGRM.mtx.sampleIDs.txt")
    write_sparse_grm(g, p.sample_ids, mtx, ids)
    return g, used, mtx, ids
