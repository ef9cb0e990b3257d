"""Regenerate the golden fixtures under tests/golden/ from the frhl/CSAIGE tree.

Usage: python make_golden.py <path of the frhl/CSAIGE tree>.  Writes:
  plink1000_500.bed/.frq  — the first 500 markers of
      extdata/input/plinkforGRM_1000samples_10kMarkers.{bed,frq}
      (1000 samples, no missing calls; PLINK's own MAF column pins the
      integer-exact allele counts);
  decode_kat.json         — the 2-bit decode known answers of
      saige-geno/src/plink.rs:288-303, transcribed as data.
"""
import argparse
import json
from pathlib import Path

HERE = Path(__file__).resolve().parent
N_MARKERS = 500


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("reference", type=Path, help="root of the frhl/CSAIGE source tree")
    ref = ap.parse_args().reference
    BASE = ref / "extdata/input/plinkforGRM_1000samples_10kMarkers"
    n_fam = sum(1 for _ in open(BASE.with_suffix(".fam")))
    bpm = (n_fam + 3) // 4
    bed = BASE.with_suffix(".bed").read_bytes()
    (HERE / "plink1000_500.bed").write_bytes(bed[: 3 + bpm * N_MARKERS])
    frq = BASE.with_suffix(".frq").read_text().splitlines()
    (HERE / "plink1000_500.frq").write_text("\n".join(frq[: 1 + N_MARKERS]) + "\n")
    kat = {
        "source": "saige-geno/src/plink.rs:288-303",
        "single": [[0b00, 0, 2.0], [0b01, 0, None], [0b10, 0, 1.0], [0b11, 0, 0.0]],
        "byte": 0b11100100,
        "offsets": [[0, 2.0], [1, None], [2, 1.0], [3, 0.0]],
        "n_fam": n_fam,
    }
    (HERE / "decode_kat.json").write_text(json.dumps(kat, indent=1) + "\n")


if __name__ == "__main__":
    main()
