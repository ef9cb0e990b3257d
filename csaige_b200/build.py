"""Build the sm_100a fit-null library in-tree: csaige_b200/libsaige_gpu.so.

Every CUDA source is compiled with nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) and linked into one shared
library with a plain C ABI (include/saige_gpu.h).  Incremental: an object is
rebuilt when its source or any header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libsaige_gpu.so"

SOURCES = [
    "engine.cu",
    "ai_reml.cu",
    "gen.cu",
    "kernels_bed.cu",
    "kernels_fp32.cu",
    "kernels_vec.cu",
    "kernels_tc.cu",
    "noalloc.cu",
    "vr.cu",
    "model.cu",
    "grm_explicit.cu",
    "warm.cu",
    "mlp.cu",
    "cohorts.cu",
    "miss_lists.cu",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the sm_100a library cannot be built")


def _host_compiler() -> list[str]:
    # The image's plain `g++` is a wrapper; prefer the versioned compiler.
    for cand in ("g++-13", "g++-12", "g++"):
        p = shutil.which(cand)
        if p:
            return ["-ccbin", p]
    return []


def _flags(verbose_ptxas: bool) -> list[str]:
    f = ARCH + [
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "--expt-relaxed-constexpr",
        "-Xcompiler",
        "-fPIC,-fvisibility=hidden,-O3",
        "-I",
        str(ROOT / "include"),
    ]
    if verbose_ptxas:
        f += ["-Xptxas", "-v"]
    return f + _host_compiler()


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def build(force: bool = False, verbose: bool = False, verbose_ptxas: bool = False) -> Path:
    nvcc = _nvcc()
    OBJ.mkdir(exist_ok=True)
    hdr = _headers_mtime()
    flags = _flags(verbose_ptxas)

    def compile_one(src: str) -> tuple[str, str]:
        s = CSRC / src
        o = OBJ / (src + ".o")
        if not force and o.exists() and o.stat().st_mtime >= max(s.stat().st_mtime, hdr):
            return src, ""
        cmd = [nvcc, *flags, "-c", str(s), "-o", str(o)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        return src, (r.stdout + r.stderr)

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        outs = list(ex.map(compile_one, SOURCES))
    if verbose or verbose_ptxas:
        for src, log in outs:
            if log.strip():
                print(f"== {src}\n{log}", file=sys.stderr)
    objs = [str(OBJ / (s + ".o")) for s in SOURCES]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcuda"] + _host_compiler()
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, verbose_ptxas="--ptxas" in sys.argv)
    print(LIB)
