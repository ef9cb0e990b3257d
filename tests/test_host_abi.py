"""Host-side checks of the C-ABI library that need no GPU: it loads, exports
every symbol include/saige_gpu.h declares, and its host-only logic matches
the oracle.  Compute calls are not made here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import csaige_b200 as cs
from csaige_b200 import _lib
import oracle_ffi as O

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    txt = (ROOT / "include" / "saige_gpu.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(saige_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert len(names) >= 15
    lib = C.CDLL(str(_lib.LIB_PATH))
    for nm in names:
        assert hasattr(lib, nm), nm
        assert nm in _lib.SIGNATURES, f"{nm} has no ctypes signature"


def test_version_and_error_string():
    assert cs.version() >= 10000
    assert isinstance(_lib.LIB.saige_last_error(), bytes)


def _synthetic_stats(m, seed):
    rng = np.random.default_rng(seed)
    n = 5000
    nv = n - rng.integers(0, 900, m)
    alt = np.array([rng.integers(0, 2 * k + 1) for k in nv])
    af = alt / (2.0 * nv)
    mac = np.minimum(alt, 2.0 * nv - alt)
    return af, mac.astype(float), nv, n


@pytest.mark.parametrize("seed", [12345, 1, 99])
def test_select_grm_markers_matches_oracle(seed):
    af, mac, nv, n = _synthetic_stats(4000, seed)
    g, v = cs.select_grm_markers(af, mac, nv, n, 0.01, 0.15, seed)
    og, ov = O.select_markers(af, mac, nv, n, 0.01, 0.15, seed)
    assert np.array_equal(g, og) and np.array_equal(v, ov)
    assert len(v) > 0 and len(set(g) & set(v)) == 0


def test_select_grm_markers_fixture(golden_dir):
    bed = np.fromfile(golden_dir / "plink1000_500.bed", dtype=np.uint8)
    af, mac, nv = O.marker_stats(bed, 1000, 500)
    g, v = cs.select_grm_markers(af, mac, nv, 1000)
    og, ov = O.select_markers(af, mac, nv, 1000)
    assert np.array_equal(g, og) and np.array_equal(v, ov)


def test_select_grm_markers_none_pass():
    with pytest.raises(cs.SaigeError) as e:
        cs.select_grm_markers([0.0, 1.0], [0.0, 0.0], [10, 10], 10)
    assert e.value.code == _lib.EINVAL


def test_bed_header_errors_need_no_gpu(golden_dir):
    bed = np.fromfile(golden_dir / "plink1000_500.bed", dtype=np.uint8)
    bad = bed.copy()
    bad[2] = 0
    with pytest.raises(cs.SaigeError) as e:
        cs.bed_marker_stats(bad, 1000, 500)
    assert e.value.code == _lib.EBED
    with pytest.raises(cs.SaigeError) as e:
        cs.bed_marker_stats(bed, 1000, 501)
    assert e.value.code == _lib.EBED


def test_generator_host_is_deterministic():
    spec = cs.CohortSpec(n=777, m=64, seed=5, cousin_frac=0.02)
    a, b = cs.gen_bed(spec), cs.gen_bed(spec)
    assert np.array_equal(a, b) and a[:3].tolist() == [0x6C, 0x1B, 0x01]
    af, mac, nv = O.marker_stats(a, 777, 64)
    miss = 1 - nv / 777
    assert 0.0 <= miss.mean() < 0.03
    y, x = cs.gen_pheno(cs.CohortSpec(n=4000, m=200, prevalence=0.1))
    assert 0.05 < y.mean() < 0.15 and x.shape == (4000, 3) and np.all(x[:, 0] == 1)


@pytest.mark.skipif(cs.device_count() > 0, reason="a GPU is present")
def test_compute_fails_loudly_without_gpu(golden_dir):
    bed = np.fromfile(golden_dir / "plink1000_500.bed", dtype=np.uint8)
    with pytest.raises(cs.SaigeError) as e:
        cs.bed_marker_stats(bed, 1000, 500)
    assert e.value.code == _lib.ECUDA


def test_ctypes_structures_match_the_header(tmp_path):
    # every struct of include/saige_gpu.h against its ctypes mirror: size and the offset
    # of each field, as gcc lays the C struct out (a mismatch would let the library
    # write past a caller's struct)
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    pairs = {"saige_pcg_options": _lib.PcgOptions, "saige_ai_reml_config": _lib.AiRemlConfigC,
             "saige_ai_reml_summary": _lib.AiRemlSummaryC,
             "saige_explicit_grm_config": _lib.ExplicitGrmConfigC,
             "saige_explicit_grm_info": _lib.ExplicitGrmInfoC,
             "saige_vr_config": _lib.VrConfigC, "saige_vr_summary": _lib.VrSummaryC,
             "saige_null_model": _lib.NullModelC, "saige_grm_stats": _lib.GrmStatsC,
             "saige_cohort_spec": _lib.CohortSpecC}
    header = Path(__file__).resolve().parents[1] / "include" / "saige_gpu.h"
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{header}"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    got = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    want = {}
    for cname, py in pairs.items():
        want[f"{cname} size"] = C.sizeof(py)
        for fname, _ in py._fields_:
            want[f"{cname} {fname}"] = getattr(py, fname).offset
    for ln in got:
        if ln:
            key, val = ln.rsplit(" ", 1)
            assert int(val) == want[key], (key, int(val), want[key])
    assert len([ln for ln in got if ln]) == len(want)
