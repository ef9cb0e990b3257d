#!/usr/bin/env python
"""fit-null benchmark on one B200 per rank.

Workload (the batched configuration of the metric): N = 200,000 samples,
M = 150,000 bed markers, binary trait at 2% prevalence, 10 covariates, 10%
sibling pairs + 2% first cousins, 1% missing calls, 30 Rademacher probes,
PCG tolerance 1e-5; synthetic cohort from the seeded generator (the
reference publishes no dataset or number for this path).

A step is one complete fit-null (GLM initialisation + AI-REML to convergence,
AiRemlConfig::default tolerances) with the genotypes resident in HBM.  The
metric is seconds per fit-null (lower is better) for the fast configuration
(MIXED int8 tensor-core GRM product, block PCG over [y, X, probes], warm
starts).  `e2e` is the same fit measured through saige_fit_null_from_bed from
pinned host buffers (bed upload, marker statistics, QC, GRM build, fit,
results back).  `plain` is one fit of the reference's own strategy (FP32
product, one PCG per right-hand side, zero starts) on the same GPU.

Under torchrun each rank fits its own cohort (independent replicas, weak
scaling); timing is the max over ranks.  `--impl reference` times the CPU
restatement of saige-rs's OnTheFlyGrm::mat_vec (oracle/, all host threads)
on a bounded marker sample and extrapolates to the fit.
"""
from __future__ import annotations

import argparse
import ctypes as C
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fit-null sec & PCG iters, N=200k M=150k: mixed+batched+learned vs plain, same GPU"
WORKLOAD = dict(n=200_000, m=150_000, prevalence=0.02, n_covar=10, sib_frac=0.10,
                cousin_frac=0.02, missing_rate=0.01, h2=0.2, seed=12345)
# GRM products (columns) of one fit of the reference's strategy on this workload
# (one PCG per right-hand side from zero, the A*0 product of each solve, and the
# 30 probe products repeated every iteration, ai_reml.rs:175-306), measured with
# the FP32 path of this library; used to extrapolate the CPU per-product time.
# Counted from a fit of this library's FP32 path with the reference strategy on the
# default workload at the fit-null command's tolerance (N=200,000, M=150,000; 5 AI-REML
# iterations, 559 PCG iterations: 559 + 5*(11+2) + 5*31 = 929, see ref_kv_count); the
# run without --no-plain recounts it on the spot.
REF_KV_PER_FIT = 929
# Markers in the bounded CPU sample (~1.6 GB of packed rows at N=200,000; about a
# second per product on 16 cores).
CPU_SAMPLE_MARKERS = 32768
# DRAM bytes read per marker row by one tensor-core launch (packed genotype tile rows
# plus the vector-limb tiles), from the ncu capture at N=200,000, m_pad=18,048:
# pass A 929.2 MB, pass B 939.4 MB.  Reads scale with m_pad; the output writes
# (pass A: m_pad*R*8 bytes, pass B: N*R*8 bytes) are added per launch.
TC_READ_PER_MARKER_ROW = {"A": 929.2e6 / 18048, "B": 939.4e6 / 18048}

FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# The plain CPU-scale fit-null cohort (the reference's own benchmark size): N = 2,000,
# M = 5,000, binary at ~10 % prevalence, 2 covariates, 10 % sibling pairs, 1 % missing.
# The precision-form cohort of the accuracy block (errors against FP64 products).
ACCURACY = dict(n=50_000, m=100_000)
# The learned-start cohort: N = 400,000, M = 100,000 (10 GB packed), binary at 1 %,
# 10 covariates, twelve AI-REML iterations.
STARTS = dict(n=400_000, m=100_000, seed=4242, iterations=12)
# tau tolerance of the fit-null command (saige-cli/src/commands/fit_null.rs:74-80)
CLI_TOL = 1e-5
CONFIG1 = dict(seed=12345, n=2000, m=5000, sib_frac=0.10, missing_rate=0.01, prevalence=0.10,
               n_covar=2, h2=0.2)
# Explicit GRM (create-sparse-grm) workload: an FP64 SYRK over all sample pairs, so
# its size is set by N^2 M / 2 products; N = 32,768 and M = 8,192 give 4.4e12.
EXPLICIT_GRM = dict(n=32_768, m=8_192, min_maf=0.01, cutoff=0.125)
# The CPU sample for it: the oracle's compute_dense_grm (reference loop order, all
# host threads) on N = 4,096 and M = 1,024 of the same cohort.
EXPLICIT_GRM_CPU = dict(n=4_096, m=1_024)
# Nominal FP64 pipe of a B200: 148 SMs x 64 FP64 lanes per clock (no measured figure
# exists for it; the clock is the one sampled during the runs).
FP64_LANES_PER_SM, N_SMS = 64, 148


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-strategy fit")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--warm", choices=["previous", "recycled", "learned"], default="recycled",
                    help="PCG start of the fast configuration")
    ap.add_argument("--no-loco", action="store_true", help="skip the LOCO fits")
    ap.add_argument("--no-cohorts", action="store_true",
                    help="skip the 16 sub-cohort fits")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the zero / recycled / learned start comparison (N=400k, M=100k)")
    ap.add_argument("--no-config1", action="store_true",
                    help="skip the plain CPU-scale cohort (GPU fits, oracle, measured CPU fit)")
    ap.add_argument("--no-plain-scale", action="store_true",
                    help="skip the plain method at GPU scale (N=50k, M=100k, quantitative)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the product and solve errors against the FP64 oracle")
    ap.add_argument("--no-explicit-grm", action="store_true",
                    help="skip the create-sparse-grm workload")
    ap.add_argument("--explicit-grm-only", action="store_true",
                    help="run only the create-sparse-grm workload and print its block")
    ap.add_argument("--grm-n", type=int, default=EXPLICIT_GRM["n"])
    ap.add_argument("--grm-m", type=int, default=EXPLICIT_GRM["m"])
    ap.add_argument("--grm-reps", type=int, default=4, help="runs per arithmetic, first untimed")
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--m", type=int, default=WORKLOAD["m"])
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return dict(FALLBACK_PEAKS), "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
            return self
        # nvidia-smi takes a moment to print its first sample: wait for it (up to 5 s) and
        # drop it, so that a short timed region is still sampled and only under load
        t0 = time.monotonic()
        while not self.lines and self.proc.poll() is None and time.monotonic() - t0 < 5.0:
            time.sleep(0.02)
        self.lines.clear()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def single_column_modes(grm, n: int, reps: int = 4) -> dict:
    """Device ms per one-column product on the bench's handle (after its timed fits) with
    the dense missing-flag sums (SAIGE_SR_LISTS=0) and with the missing-call lists the
    handle built in its second warm-up fit: the same products to the bit."""
    import numpy as np

    v = np.random.default_rng(3).standard_normal((1, n))
    prev = os.environ.get("SAIGE_SR_LISTS")
    out = {}
    grm.set_profiling(True)
    try:
        for mode, key in (("0", "flags"), ("1", "lists")):
            os.environ["SAIGE_SR_LISTS"] = mode
            grm.mat_vec(v)
            grm.reset_stats()
            for _ in range(reps):
                grm.mat_vec(v)
            s = grm.stats()
            out[key + "_ms"] = s["sc_ms"] / max(s["sc_launches"], 1)
            out[key + "_list_products"] = s["sc_list_launches"]
    finally:
        if prev is None:
            os.environ.pop("SAIGE_SR_LISTS", None)
        else:
            os.environ["SAIGE_SR_LISTS"] = prev
        grm.set_profiling(False)
    out["products"] = reps
    return out


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(x: float, world: int, device: str) -> float:
    """Maximum of x over all ranks (device "cuda" under NCCL, "cpu" under gloo)."""
    if world == 1:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def whole_job_seconds_per_fit(step_max_s: float, world: int) -> float:
    """N replicas each fit their own cohort in one step: the job completes N fits
    in the slowest rank's step time."""
    return step_max_s / world


def ref_kv_count(iterations: int, p: int, nrv: int, pcg_iters: int, solves_per_iter: int) -> int:
    """GRM products of the reference strategy: PCG iterations, one A*0 product
    per solve, and K*Py plus the probe products every iteration."""
    return pcg_iters + iterations * solves_per_iter + iterations * (1 + nrv)


# ---------------------------------------------------------------------------
# reference arm: CPU restatement, bounded marker sample, extrapolated
# ---------------------------------------------------------------------------
class CpuSample:
    """The oracle's packed f32 OnTheFlyGrm::mat_vec (saige-core/src/glmm/pcg.rs:128-180
    arithmetic, per-thread fold, all host threads) on `markers` synthetic markers of
    the workload's cohort; products are timed and extrapolated to m_full markers.
    The cohort comes from the oracle's statement of the generator, so nothing of the
    library is loaded."""

    def __init__(self, n: int, markers: int):
        sys.path.insert(0, str(ROOT / "tests"))
        import numpy as np

        import oracle_ffi as O

        O.L.orc_grm_matvec_f32_packed.restype = C.c_int
        O.L.orc_grm_matvec_f32_packed.argtypes = [C.POINTER(C.c_uint8), C.c_int64, C.c_int64,
                                                  C.POINTER(C.c_int64), C.c_int64, O._d, O._d,
                                                  O._d, C.c_int]
        self.O, self.np = O, np
        self.n, self.markers = n, markers
        spec = O.cohort_spec(n=n, m=markers, seed=WORKLOAD["seed"], sib_frac=WORKLOAD["sib_frac"],
                             cousin_frac=WORKLOAD["cousin_frac"],
                             missing_rate=WORKLOAD["missing_rate"])
        bed = O.gen_bed(spec)
        self.af, _, _ = O.marker_stats(bed, n, markers)
        self.body = np.ascontiguousarray(bed[3:])
        self.rows = np.arange(markers, dtype=np.int64)
        self.v = np.random.default_rng(1).standard_normal(n)
        self.out = np.empty(n)
        self.threads = 0

    def product_seconds(self) -> float:
        """Seconds of one product over the sample."""
        O = self.O
        t0 = time.perf_counter()
        self.threads = O.L.orc_grm_matvec_f32_packed(
            self.body.ctypes.data_as(C.POINTER(C.c_uint8)), (self.n + 3) // 4, self.n,
            self.rows.ctypes.data_as(C.POINTER(C.c_int64)), self.markers, O.dp(self.af),
            O.dp(self.v), O.dp(self.out), 0)
        return time.perf_counter() - t0

    def describe(self, m_full: int, kv_fit: int) -> str:
        return (f"OnTheFlyGrm::mat_vec arithmetic (f32, per-thread fold) on {self.markers} of "
                f"{m_full} markers x {self.n} samples, extrapolated x{m_full / self.markers:.1f} "
                f"per product and x{kv_fit} products per fit (reference strategy count)")


def cpu_config1_fit() -> dict:
    """A whole fit-null measured on the host cores, not extrapolated: the plain cohort
    (N = 2,000, M = 5,000, binary ~10 %, 2 covariates, seed 12345) from .bed bytes to
    tau with the oracle — marker statistics, QC and the VR/GRM split, f32 Z
    (pcg.rs:101-122) and fit_ai_reml (ai_reml.rs:86-427) at the fit-null command's
    settings (tol 1e-5, max_iter 30) with the f32 product on all threads (the rayon
    fold and reduce of pcg.rs:149-176)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ffi as O

    spec = O.cohort_spec(**CONFIG1)
    bed = O.gen_bed(spec)
    y, x = O.gen_pheno(spec)
    t0 = time.perf_counter()
    af, mac, nv = O.marker_stats(bed, spec.n, spec.m)
    g, _ = O.select_markers(af, mac, nv, spec.n)
    z = O.standardize(O.dosages(bed, spec.n, g), af[g], 1)
    t1 = time.perf_counter()
    o = O.fit_ai_reml(y, x, O.BINARY, O.K_OTF, z, m=len(g), kmode=2, max_iter=30, tol=1e-5)
    t2 = time.perf_counter()
    return {"workload": "fit-null binary ~10% prev, N=2000, M=5000, 2 covariates, 30 probes, "
                        "tol 1e-5 (measured whole fit, oracle f32 product on all host threads)",
            "pipeline_s": t2 - t0, "fit_s": t2 - t1, "cores": os.cpu_count(),
            "tau": [float(o["tau"][0]), float(o["tau"][1])], "iterations": int(o["iterations"]),
            "n_kv": int(o["n_kv"]), "pcg_iters": int(o["pcg_iters"]), "markers_grm": int(len(g))}


def explicit_grm_block(cs, gpu_index: int, n: int, m: int, reps: int = 4,
                       cpu: bool = True) -> dict:
    """compute_sparse_grm (saige-core/src/grm/sparse.rs:18-66) from host .bed bytes to
    the sorted sparse triplets, on EXPLICIT_GRM; kernel time from the library's CUDA
    events, e2e from the call's own clock; the CPU oracle on a bounded sample."""
    g = dict(EXPLICIT_GRM, n=n, m=m)
    spec = cs.CohortSpec(n=g["n"], m=g["m"], seed=WORKLOAD["seed"], sib_frac=WORKLOAD["sib_frac"],
                         cousin_frac=WORKLOAD["cousin_frac"],
                         missing_rate=WORKLOAD["missing_rate"])
    bed = cs.gen_bed(spec)
    out = {"workload": (f"create-sparse-grm: N={g['n']} samples, M={g['m']} markers "
                        f"(the fit-null cohort generator), min_maf {g['min_maf']}, "
                        f"cutoff {g['cutoff']}, host .bed in, sorted triplets out")}
    with ClockSampler(gpu_index) as clk:
        for arith, key in ((cs.GRM_ARITH_REFERENCE, "reference_arith"),
                           (cs.GRM_ARITH_FMA, "fma_arith")):
            ks, tot = [], []
            for rep in range(max(reps, 2)):  # the first is a warm-up
                sp, used = cs.compute_sparse_grm(bed, g["n"], g["m"], g["min_maf"], g["cutoff"],
                                                 arith=arith)
                if rep:
                    ks.append(sp.info.kernel_seconds)
                    tot.append(sp.info.total_seconds)
            k = statistics.median(ks)
            out[key] = {"kernel_s": k, "e2e_s": statistics.median(tot),
                        "terms_per_s": sp.info.terms / k}
    c = clk.summary()
    mhz = c["sm_mhz"] or c["sm_max_mhz"] or 1965.0
    peak_ops = N_SMS * FP64_LANES_PER_SM * mhz * 1e6
    # reference arithmetic: a DMUL and a DADD per product; FMA: one DFMA
    out["reference_arith"]["fp64_pipe_frac"] = 2 * out["reference_arith"]["terms_per_s"] / peak_ops
    out["fma_arith"]["fp64_pipe_frac"] = out["fma_arith"]["terms_per_s"] / peak_ops
    out.update({"terms": sp.info.terms, "n_markers_used": int(used), "nnz": int(sp.vals.size),
                "fp64_peak": f"nominal {N_SMS} SMs x {FP64_LANES_PER_SM} lanes at {mhz:.0f} MHz",
                "clocks": c, "parity": "reference_arith bit-identical to the oracle (tests)"})
    if not cpu:
        return out
    # CPU: the oracle in the reference's loop order on a bounded sample
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_ffi as O
    cg = EXPLICIT_GRM_CPU
    cbed = cs.gen_bed(cs.CohortSpec(n=cg["n"], m=cg["m"], seed=WORKLOAD["seed"],
                                    sib_frac=WORKLOAD["sib_frac"],
                                    cousin_frac=WORKLOAD["cousin_frac"],
                                    missing_rate=WORKLOAD["missing_rate"]))
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        _, cu = O.dense_grm_bed(cbed, cg["n"], cg["m"], g["min_maf"])
        times.append(time.perf_counter() - t0)
    rate = cg["n"] * (cg["n"] + 1) / 2 * cu / min(times)
    out["cpu_baseline"] = {"terms_per_s": rate, "cores": os.cpu_count(), "kind": "port",
                           "sample": f"oracle compute_dense_grm on N={cg['n']}, M={cg['m']}",
                           "extrapolated_s": sp.info.terms / rate}
    out["speedup_e2e_vs_cpu"] = out["cpu_baseline"]["extrapolated_s"] / out["reference_arith"]["e2e_s"]
    return out


def config1_block(cs) -> dict:
    """The plain CPU-scale cohort (N = 2,000, M = 5,000): the fast and the plain GPU fits
    at the command's tolerance, tau against the FP64 oracle (exact GRM), and a whole
    CPU fit measured beside them."""
    sys.path.insert(0, str(ROOT / "tests"))
    import numpy as np

    import oracle_ffi as O

    spec = cs.CohortSpec(**CONFIG1)
    bed = cs.gen_bed(spec)
    y, x = cs.gen_pheno(spec)
    af, mac, nv = cs.bed_marker_stats(bed, spec.n, spec.m)
    g, _ = cs.select_grm_markers(af, mac, nv, spec.n)
    out = {"workload": "fit-null binary ~10% prev, N=2000, M=5000, 2 covariates, 30 probes, "
                       "tol 1e-5"}
    k = O.grm_explicit(O.standardize(O.dosages(bed, spec.n, g), af[g], 0))
    o = O.fit_ai_reml(y, x, O.BINARY, O.K_EXPLICIT, k, max_iter=30, tol=CLI_TOL)
    out["oracle_fp64_tau"] = [float(o["tau"][0]), float(o["tau"][1])]
    for name, prec, solve, warm in (("fast", cs.PREC_MIXED, cs.SOLVE_BLOCK, cs.WARM_RECYCLED),
                                    ("plain", cs.PREC_FP32, cs.SOLVE_SINGLE, cs.WARM_ZERO)):
        grm = cs.OnTheFlyGrm.from_bed(bed, spec.n, spec.m, g, af[g], precision=prec)
        cfg = cs.AiRemlConfig(precision=prec, solve=solve, warm_start=warm, tol=CLI_TOL,
                              max_iter=30)
        cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg)  # warm-up
        rs = [cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg) for _ in range(3)]
        r = rs[-1]
        out[name] = {"seconds": statistics.median(q.seconds for q in rs),
                     "ai_reml_iterations": int(r.iterations), "n_kv": int(r.n_kv),
                     "n_kv_launches": int(r.n_kv_launches), "pcg_iters": int(r.pcg_iters),
                     "tau": [float(r.tau[0]), float(r.tau[1])],
                     "tau_rel_err_vs_fp64_oracle": float(abs(r.tau[1] - o["tau"][1]) /
                                                         abs(o["tau"][1]))}
        grm.close()
    out["cpu_fit"] = cpu_config1_fit()
    out["speedup_fast_vs_cpu_fit"] = out["cpu_fit"]["fit_s"] / out["fast"]["seconds"]
    return out


def accuracy_block(cs) -> dict:
    """The precision-form cohort (N = 50,000, M = 100,000, binary at 5 %, 6
    covariates): errors of the GPU products against the oracle's FP64 product on the
    same packed genotypes, and the true residual of Sigma^-1 y (FP64 products) at the
    fast fit's tau and W."""
    sys.path.insert(0, str(ROOT / "tests"))
    import numpy as np
    import torch

    import oracle_ffi as O

    n, m = ACCURACY["n"], ACCURACY["m"]
    spec = cs.CohortSpec(n=n, m=m, seed=WORKLOAD["seed"], sib_frac=WORKLOAD["sib_frac"],
                         cousin_frac=WORKLOAD["cousin_frac"], missing_rate=WORKLOAD["missing_rate"],
                         trait=cs.TraitType.Binary, n_covar=6, prevalence=0.05, h2=0.2,
                         n_causal=1000)
    bed_dev = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, bed_dev.data_ptr())
    bed = bed_dev.cpu().numpy()
    y, x = cs.gen_pheno(spec)
    af, mac, nv = cs.api.bed_marker_stats_dev(bed_dev.data_ptr(), spec.bed_len, n, m)
    g, _ = cs.select_grm_markers(af, mac, nv, n)
    grm = cs.OnTheFlyGrm.from_bed_dev(bed_dev.data_ptr(), spec.bed_len, n, m, g, af[g],
                                      precision=cs.PREC_MIXED)
    del bed_dev
    torch.cuda.empty_cache()
    rng = np.random.default_rng(7)
    v = np.vstack([rng.standard_normal(n), y - y.mean(), O.probes(12345, 1, n)[0]])
    want = O.grm_matmul_f64_packed(bed, n, g, af[g], v)

    def errs(got):
        return {"max_rel": float(max(np.abs(got[c] - want[c]).max() / np.abs(want[c]).max()
                                     for c in range(len(v)))),
                "l2_rel": float(max(np.linalg.norm(got[c] - want[c]) / np.linalg.norm(want[c])
                                    for c in range(len(v))))}

    out = {"workload": f"binary 5% prev, N={n}, M={m} bed markers ({len(g)} in the GRM), "
                       f"6 covariates; errors against the oracle's FP64 product",
           "kv_columns": "N(0,1), y - mean(y), a Rademacher probe",
           "kv_mixed_tensor_cores": errs(grm.mat_vec(v, precision=cs.PREC_MIXED)),
           "kv_mixed_one_column": errs(np.vstack([grm.mat_vec(v[c], precision=cs.PREC_MIXED)
                                                  for c in range(len(v))])),
           "kv_fp32": errs(grm.mat_vec(v, precision=cs.PREC_FP32))}
    fits = {}
    for name, prec, solve, warm in (("fast", cs.PREC_MIXED, cs.SOLVE_BLOCK, cs.WARM_RECYCLED),
                                    ("plain", cs.PREC_FP32, cs.SOLVE_SINGLE, cs.WARM_ZERO)):
        cfg = cs.AiRemlConfig(precision=prec, solve=solve, warm_start=warm, tol=CLI_TOL,
                              max_iter=30)
        r = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg)
        fits[name] = r
        sol = cs.PcgSolver(1e-5, 500).solve(grm, r.working_weights, r.tau, y, precision=prec)
        kx = O.grm_matmul_f64_packed(bed, n, g, af[g], sol.x)
        sig_x = r.tau[0] * sol.x / np.maximum(r.working_weights, 1e-30) + r.tau[1] * kx
        out[f"{name}_fit"] = {
            "seconds": r.seconds, "ai_reml_iterations": int(r.iterations),
            "tau": [float(r.tau[0]), float(r.tau[1])], "pcg_iters": int(r.pcg_iters),
            "sigma_inv_y_true_residual": float(np.linalg.norm(y - sig_x) / np.linalg.norm(y)),
            "sigma_inv_y_pcg_iters": int(sol.iterations)}
    out["tau_rel_diff_fast_vs_plain"] = float(abs(fits["fast"].tau[1] - fits["plain"].tau[1]) /
                                              abs(fits["plain"].tau[1]))
    out["note"] = ("tau against an FP64 fit is checked on the CPU-scale cohort (config1 block "
                   "and the tests); here the FP64 oracle provides the products")
    grm.close()
    return out


def plain_scale_block(cs) -> dict:
    """The plain method at GPU scale (N = 50,000, M = 100,000, a quantitative trait with
    h2 = 0.3, 4 N(0,1) covariates, Gaussian noise, 30 probes, tolerance 1e-5): the
    reference's strategy (FP32 products, one PCG per right-hand side, zero starts) and
    the fast configuration on the same cohort, each with seconds, iterations, tau, and
    the true residual of Sigma^-1 y with the oracle's FP64 products at its own tau and W;
    plus the FP32 product's error against the FP64 product."""
    sys.path.insert(0, str(ROOT / "tests"))
    import numpy as np
    import torch

    import oracle_ffi as O

    n, m = ACCURACY["n"], ACCURACY["m"]
    spec = cs.CohortSpec(n=n, m=m, seed=WORKLOAD["seed"] + 1, sib_frac=WORKLOAD["sib_frac"],
                         cousin_frac=WORKLOAD["cousin_frac"], missing_rate=WORKLOAD["missing_rate"],
                         trait=cs.TraitType.Quantitative, n_covar=4, h2=0.3)
    bed_dev = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, bed_dev.data_ptr())
    bed = bed_dev.cpu().numpy()
    y, x = cs.gen_pheno(spec)
    af, mac, nv = cs.api.bed_marker_stats_dev(bed_dev.data_ptr(), spec.bed_len, n, m)
    g, _ = cs.select_grm_markers(af, mac, nv, n)
    out = {"workload": f"quantitative h2 0.3, N={n}, M={m} bed markers ({len(g)} in the GRM), "
                       f"4 covariates, 30 probes, tol 1e-5"}
    fits = {}
    for name, prec, solve, warm in (("plain", cs.PREC_FP32, cs.SOLVE_SINGLE, cs.WARM_ZERO),
                                    ("fast", cs.PREC_MIXED, cs.SOLVE_BLOCK, cs.WARM_RECYCLED)):
        grm = cs.OnTheFlyGrm.from_bed_dev(bed_dev.data_ptr(), spec.bed_len, n, m, g, af[g],
                                          precision=prec)
        if name == "plain":
            v = np.random.default_rng(7).standard_normal(n)
            want = O.grm_matmul_f64_packed(bed, n, g, af[g], v[None, :])[0]
            got = grm.mat_vec(v, precision=cs.PREC_FP32)
            out["kv_fp32_max_rel"] = float(np.abs(got - want).max() / np.abs(want).max())
        cfg = cs.AiRemlConfig(precision=prec, solve=solve, warm_start=warm, tol=CLI_TOL,
                              max_iter=30)
        r = cs.fit_ai_reml(y, x, grm, cs.TraitType.Quantitative, cfg)
        fits[name] = r
        sol = cs.PcgSolver(1e-5, 500).solve(grm, r.working_weights, r.tau, y, precision=prec)
        kx = O.grm_matmul_f64_packed(bed, n, g, af[g], sol.x[None, :])[0]
        sig_x = r.tau[0] * sol.x / np.maximum(r.working_weights, 1e-30) + r.tau[1] * kx
        out[f"{name}_fit"] = {
            "seconds": r.seconds, "ai_reml_iterations": int(r.iterations),
            "n_kv": int(r.n_kv), "n_kv_launches": int(r.n_kv_launches),
            "pcg_iters": int(r.pcg_iters), "tau": [float(r.tau[0]), float(r.tau[1])],
            "sigma_inv_y_true_residual": float(np.linalg.norm(y - sig_x) / np.linalg.norm(y))}
        grm.close()
    del bed_dev
    torch.cuda.empty_cache()
    out["tau_rel_diff_fast_vs_plain"] = float(max(
        abs(fits["fast"].tau[k] - fits["plain"].tau[k]) / abs(fits["plain"].tau[k])
        for k in (0, 1)))
    out["speedup_fast_vs_plain"] = fits["plain"].seconds / fits["fast"].seconds
    return out


def starts_block(cs) -> dict:
    """The learned-start cohort (N = 400,000, M = 100,000, binary at 1 %, 10
    covariates): twelve AI-REML iterations of the fast configuration (MIXED, block PCG
    to 1e-5, the reference's diagonal preconditioner) from the zero, the recycled and
    the learned start; products launched, PCG iterations and seconds of each."""
    import torch

    n, m = STARTS["n"], STARTS["m"]
    spec = cs.CohortSpec(n=n, m=m, seed=STARTS["seed"], sib_frac=WORKLOAD["sib_frac"],
                         cousin_frac=WORKLOAD["cousin_frac"], missing_rate=WORKLOAD["missing_rate"],
                         trait=cs.TraitType.Binary, n_covar=10, prevalence=0.01, h2=0.2,
                         n_causal=1000)
    bed_dev = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, bed_dev.data_ptr())
    y, x = cs.gen_pheno(spec)
    af, mac, nv = cs.api.bed_marker_stats_dev(bed_dev.data_ptr(), spec.bed_len, n, m)
    g, _ = cs.select_grm_markers(af, mac, nv, n)
    grm = cs.OnTheFlyGrm.from_bed_dev(bed_dev.data_ptr(), spec.bed_len, n, m, g, af[g],
                                      precision=cs.PREC_MIXED)
    del bed_dev
    torch.cuda.empty_cache()
    out = {"workload": f"fit-null binary 1% prev (cases {int(y.sum())}), N={n}, M={m} bed "
                       f"markers ({len(g)} in the GRM), 10 covariates, 30 probes, PCG tol 1e-5, "
                       f"{STARTS['iterations']} AI-REML iterations (tau tolerance 0)",
           "config": "MIXED tensor-core products, block PCG over y, X and the probes, "
                     "diagonal (tau0/W + tau1) preconditioner"}
    for name, wmode in (("zero", cs.WARM_ZERO), ("recycled", cs.WARM_RECYCLED),
                        ("learned", cs.WARM_LEARNED)):
        cfg = cs.AiRemlConfig(precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK, warm_start=wmode,
                              tol=0.0, max_iter=STARTS["iterations"])
        t0 = time.perf_counter()
        r = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cfg)
        wall = time.perf_counter() - t0
        out[name] = {"seconds": r.seconds, "wall_s": wall, "ai_reml_iterations": int(r.iterations),
                     "n_kv_launches": int(r.n_kv_launches), "n_kv": int(r.n_kv),
                     "pcg_iters": int(r.pcg_iters), "tau": [float(r.tau[0]), float(r.tau[1])]}
        if wmode == cs.WARM_LEARNED:
            out[name].update({"trainings": int(r.learned_trainings),
                              "prediction_used": int(r.learned_uses),
                              "held_out_r2": float(r.learned_r2),
                              "mlp_seconds": float(r.learned_seconds)})
    for name in ("recycled", "learned"):
        out[f"{name}_vs_zero"] = {
            "launches_saved": out["zero"]["n_kv_launches"] - out[name]["n_kv_launches"],
            "pcg_iters_saved": out["zero"]["pcg_iters"] - out[name]["pcg_iters"],
            "speedup": out["zero"]["seconds"] / out[name]["seconds"]}
    out["learned_vs_recycled"] = {
        "launches_saved": out["recycled"]["n_kv_launches"] - out["learned"]["n_kv_launches"],
        "pcg_iters_saved": out["recycled"]["pcg_iters"] - out["learned"]["pcg_iters"],
        "speedup": out["recycled"]["seconds"] / out["learned"]["seconds"],
        "tau_rel_diff": abs(out["learned"]["tau"][1] - out["recycled"]["tau"][1]) /
                        abs(out["recycled"]["tau"][1])}
    grm.close()
    return out


def run_reference(args, rank):
    """The reference's strategy on the host cores: each step times one product of the
    oracle over a bounded marker sample and extrapolates it to a whole fit at the
    benchmark size (labelled extrapolated); a whole fit of the plain CPU-scale cohort
    is measured once beside it.  Only the oracle is loaded."""
    if rank != 0:
        return
    smp = CpuSample(args.n, min(CPU_SAMPLE_MARKERS, args.m))
    steps = []
    for _ in range(args.warmup + args.steps):
        per_kv = smp.product_seconds() * args.m / smp.markers
        steps.append(per_kv * REF_KV_PER_FIT)
    timed = steps[args.warmup:]
    val = statistics.median(timed)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": val * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": _config(args),
        "cpu_baseline": {"value": val, "unit": "s", "cores": smp.threads, "kind": "port",
                         "sample": smp.describe(args.m, REF_KV_PER_FIT), "extrapolated": True,
                         "sec_per_kv": val / REF_KV_PER_FIT},
        "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "cpu_fit_config1": cpu_config1_fit(),
    }
    print(json.dumps(line), flush=True)


def _config(args):
    return {"workload": f"fit-null binary 2% prev, N={args.n} samples, M={args.m} markers, "
                        f"10 covariates, 30 probes, PCG tol 1e-5",
            "samples": args.n, "markers": args.m, "rhs_block": 1 + 11 + 30,
            "parallelism": f"replicas x{args.gpus}",
            "l2": "inputs larger than L2 (packed genotypes 7.5 GB)"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import csaige_b200 as cs

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    n, m = args.n, args.m
    spec = cs.CohortSpec(n=n, m=m, seed=WORKLOAD["seed"] + rank, sib_frac=WORKLOAD["sib_frac"],
                         cousin_frac=WORKLOAD["cousin_frac"],
                         missing_rate=WORKLOAD["missing_rate"], trait=cs.TraitType.Binary,
                         n_covar=WORKLOAD["n_covar"], prevalence=WORKLOAD["prevalence"],
                         h2=WORKLOAD["h2"], n_causal=1000)
    bed_dev = torch.empty(spec.bed_len, dtype=torch.uint8, device="cuda")
    cs.gen_bed_dev(spec, bed_dev.data_ptr())
    torch.cuda.synchronize()
    y, x = cs.gen_pheno(spec)
    p = x.shape[1]
    af, mac, nv = cs.api.bed_marker_stats_dev(bed_dev.data_ptr(), spec.bed_len, n, m)
    gidx, vidx = cs.select_grm_markers(af, mac, nv, n, 0.01, 0.15, 12345)
    grm = cs.OnTheFlyGrm.from_bed_dev(bed_dev.data_ptr(), spec.bed_len, n, m, gidx, af[gidx],
                                      precision=cs.PREC_MIXED)
    host_bed = None
    if not args.no_e2e:
        host_bed = torch.empty(spec.bed_len, dtype=torch.uint8, pin_memory=True)
        host_bed.copy_(bed_dev)
    del bed_dev
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    warm = {"previous": cs.WARM_PREVIOUS, "recycled": cs.WARM_RECYCLED,
            "learned": cs.WARM_LEARNED}[args.warm]
    # the fit-null command's settings (fit_null.rs:74-80, 273-282): tau tolerance 1e-5,
    # 30 AI-REML iterations at most, PCG tolerance 1e-5
    fast = cs.AiRemlConfig(precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK, warm_start=warm,
                           tol=CLI_TOL, max_iter=30)
    for _ in range(args.warmup):
        cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, fast)
    grm.reset_stats()
    grm.set_profiling(True)
    l0 = cs.kernel_launches()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    results = []
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            results.append(cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, fast))
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if world > 1:
        torch.distributed.barrier()
    launches = cs.kernel_launches() - l0
    st = grm.stats()
    grm.set_profiling(False)
    dev_s = [r.seconds for r in results]
    step_s = reduce_max(statistics.mean(dev_s), world, "cuda")  # device time, max over ranks
    last = results[-1]

    # roofline of the dominant tensor-core pass, from the live CUDA-event timing
    pk, pk_kind = peaks()
    hbm = float(pk.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"]))
    bf16 = float(pk.get("bf16_tflops_sustained", pk.get("bf16_tflops", FALLBACK_PEAKS["bf16_tflops"])))
    passes = {"A": (st["tc_pass_a_ms"], st["tc_pass_a_launches"]),
              "B": (st["tc_pass_b_ms"], st["tc_pass_b_launches"])}
    dom = max(passes, key=lambda k: passes[k][0])
    tot_ms, nl = passes[dom]
    avg_s = (tot_ms / max(nl, 1)) * 1e-3
    m_grm = grm.n_markers
    # right-hand sides per tensor-core launch (single columns run on the CUDA cores)
    cols = (st["n_kv"] - st["sc_launches"]) / max(st["tc_pass_a_launches"], 1)
    bytes_launch = m_grm * ((n + 3) // 4)                # packed genotypes read once per pass
    flops_launch = 2.0 * n * m_grm * cols                 # one GEMM of an N x M by M x r product
    int8_peak_tops = 2.0 * bf16                           # dense int8 = 2x bf16 on B200
    t_hbm = bytes_launch / (hbm * 1e9)
    t_tc = flops_launch / (int8_peak_tops * 1e12)
    if t_hbm >= t_tc:
        roof = {"bound": "hbm", "achieved": bytes_launch / avg_s / 1e9, "peak": hbm, "unit": "GB/s"}
    else:
        roof = {"bound": "tensor", "achieved": flops_launch / avg_s / 1e12, "peak": int8_peak_tops,
                "unit": "TFLOP/s"}
    roof["frac"] = roof["achieved"] / roof["peak"]
    # per-launch DRAM traffic: measured read bytes per marker row scaled to this m_pad,
    # plus the launch's output writes
    m_pad = -(-m_grm // 128) * 128
    out_bytes = (m_pad if dom == "A" else n) * cols * 8
    roof["traffic"] = TC_READ_PER_MARKER_ROW[dom] * m_pad + out_bytes
    roof["kernel"] = f"tc_grm_kernel pass {dom} (MIXED, {cols:.1f} rhs per launch)"
    roof["peak_source"] = (f"{pk_kind} MEASURED_PEAKS.json" if pk_kind == "measured" else "fallback")
    roof["avg_launch_ms"] = avg_s * 1e3
    roof["share_of_step"] = (st["tc_pass_a_ms"] + st["tc_pass_b_ms"]) / 1e3 / (step_s * args.steps)
    if st["sc_launches"]:
        # one-column products (dp4a on the CUDA cores): both passes read the codes once
        sc_avg = st["sc_ms"] / st["sc_launches"] * 1e-3
        listed = st["missing_listed"]
        roof["single_column"] = {
            "kernels": ("sr_pass_a_kernel + sr_pass_b_kernel (+ quantisation)"
                        + (", summing over the missing-call lists" if st["sc_list_launches"]
                           else "")),
            "missing_lists": {"products": st["sc_list_launches"], "calls": listed,
                              "index_bytes_per_pass": 4 * listed if listed > 0 else 0},
            "products_per_step": st["sc_launches"] / args.steps, "avg_ms": sc_avg * 1e3,
            "achieved_gbs": 2 * bytes_launch / sc_avg / 1e9,
            "frac": 2 * bytes_launch / sc_avg / 1e9 / hbm,
            "share_of_step": st["sc_ms"] / 1e3 / (step_s * args.steps)}
        if world == 1:
            roof["single_column"]["flags_vs_lists"] = single_column_modes(grm, args.n)

    line = {
        "metric": METRIC, "value": whole_job_seconds_per_fit(step_s, world), "unit": "s",
        "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8 tensor products, f64 solver",
        "data": "synthetic", "config": _config(args),
        "pcg_iters": int(last.pcg_iters), "ai_reml_iterations": int(last.iterations),
        "tau": [float(last.tau[0]), float(last.tau[1])], "n_kv": int(last.n_kv),
        "n_kv_launches": int(last.n_kv_launches), "wall_s_per_step": wall / args.steps,
        "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary(),
        "markers_grm": int(m_grm), "markers_vr": int(len(vidx)),
        "fast_config": f"MIXED + block PCG + {args.warm} warm start",
    }

    # the same fit at AiRemlConfig::default's tau tolerance (0.02, ai_reml.rs:39-51)
    dcfg = dataclasses.replace(fast, tol=0.02)
    dres = [cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, dcfg) for _ in range(3)]
    line["default_tol_fit"] = {
        "tol": 0.02, "seconds": statistics.mean(r.seconds for r in dres),
        "ai_reml_iterations": int(dres[-1].iterations),
        "n_kv_launches": int(dres[-1].n_kv_launches), "pcg_iters": int(dres[-1].pcg_iters),
        "tau": [float(dres[-1].tau[0]), float(dres[-1].tau[1])]}

    # end to end through the host-buffer C ABI
    if host_bed is not None:
        hb = host_bed.numpy()
        cs.fit_null_from_bed(hb, n, m, y, x, cs.TraitType.Binary, fast)  # warm-up
        e2e_t = []
        for _ in range(min(args.steps, 2)):
            t0 = time.perf_counter()
            fr = cs.fit_null_from_bed(hb, n, m, y, x, cs.TraitType.Binary, fast)
            e2e_t.append(time.perf_counter() - t0)
        e2e_s = reduce_max(statistics.mean(e2e_t), world, "cuda")
        line["e2e"] = {"value": whole_job_seconds_per_fit(e2e_s, world), "unit": "s",
                       "h2d_bytes_per_step": int(spec.bed_len + y.nbytes + x.nbytes),
                       "d2h_bytes_per_step": int(8 * (p + n + 2 * fast.max_iter)),
                       "tau": [float(fr.ai_reml.tau[0]), float(fr.ai_reml.tau[1])]}
        # the rest of fit-null (fit_null.rs:290-373): the variance ratio over the VR
        # candidates, in the same call; reported beside the headline, not in it
        vcfg = cs.VarianceRatioConfig(precision=cs.PREC_MIXED)
        t0 = time.perf_counter()
        fv = cs.fit_null_from_bed(hb, n, m, y, x, cs.TraitType.Binary, fast, variance_ratio=True,
                                  vr_config=vcfg)
        wall_vr = time.perf_counter() - t0
        v = fv.variance_ratio
        line["variance_ratio"] = {
            "value": v.variance_ratio, "markers_used": v.n_markers_used,
            "markers_solved": v.n_solved, "blocks": v.n_blocks, "pcg_iters": int(v.pcg_iters),
            "n_kv": int(v.n_kv), "device_s": v.seconds,
            "fit_null_with_vr_wall_s": wall_vr,
            # the reference solves each used marker alone: its PCG iterations plus the
            # A*0 product of each solve (decomposition.rs:226)
            "reference_kv_estimate": int(v.pcg_iters + v.n_solved)}
    # LOCO (loco.rs:54-117): one fit per chromosome with it left out of the GRM; the
    # GRM markers are split into 22 blocks in proportion to the GRCh38 autosome lengths
    loco_sizes = None
    if not args.no_loco and world == 1:
        lengths = [248, 242, 198, 190, 181, 171, 159, 145, 138, 134, 135, 133, 114, 107, 102,
                   90, 83, 80, 59, 64, 47, 51]
        mg = len(gidx)
        cuts = (np.cumsum([0] + lengths) / sum(lengths) * mg).astype(int)
        chrom = [""] * mg
        for c in range(22):
            for j in range(cuts[c], cuts[c + 1]):
                chrom[j] = str(c + 1)
        loco_sizes = [int(cuts[c + 1] - cuts[c]) for c in range(22)]
        t0 = time.perf_counter()
        lres = cs.run_loco(y, x, grm, chrom, cs.TraitType.Binary, fast)
        lwall = time.perf_counter() - t0
        line["loco"] = {
            "chromosomes": 22, "wall_s": lwall,
            "device_s": float(sum(r.seconds for r in lres.values())),
            "n_kv": int(sum(r.n_kv for r in lres.values())),
            "ai_reml_iterations": int(sum(r.iterations for r in lres.values())),
            "config": "22 chromosome blocks of the GRM markers, fast configuration, one handle "
                      "(markers left out by masking between the product passes)"}
    # 16 sub-cohorts of the same .bed, N log-uniform in [5k, 60k] (the workload's
    # sub-cohort part): their fits one after the other and concurrently (own threads and
    # streams), from the same host buffer
    if not args.no_cohorts and world == 1 and host_bed is not None:
        rng = np.random.default_rng(WORKLOAD["seed"])
        sizes = np.exp(rng.uniform(np.log(5000), np.log(min(60000, n)), 16)).astype(int)
        cohorts = []
        for sz in sizes:
            idx = np.sort(rng.choice(n, int(sz), replace=False))
            cohorts.append((idx, y[idx], x[idx]))
        hb = host_bed.numpy()
        # one untimed call of each mode first (the device buffers of 16 handles, ~43 GB, and
        # the pinned count/row-map block are allocated once and reused by later calls)
        for conc in (False, True):
            cs.fit_null_cohorts(hb, n, m, cohorts, cs.TraitType.Binary, fast, concurrent=conc)
        # three runs of each, alternating (the wall times of 16 small host-driven fits vary
        # by ~15 % from run to run); medians reported
        seq_walls, con_walls, same = [], [], True
        for _ in range(3):
            seq, w = cs.fit_null_cohorts(hb, n, m, cohorts, cs.TraitType.Binary, fast,
                                         concurrent=False)
            seq_walls.append(w)
            con, w = cs.fit_null_cohorts(hb, n, m, cohorts, cs.TraitType.Binary, fast,
                                         concurrent=True)
            con_walls.append(w)
            same = same and all(np.array_equal(a.tau, b.tau) and a.m_grm == b.m_grm
                                for a, b in zip(seq, con))
        seq_wall, con_wall = statistics.median(seq_walls), statistics.median(con_walls)
        line["sub_cohorts"] = {
            "n_cohorts": len(cohorts), "sizes": [int(v) for v in sizes],
            "sequential_s": seq_wall, "concurrent_s": con_wall,
            "sequential_runs_s": seq_walls, "concurrent_runs_s": con_walls,
            "speedup": seq_wall / con_wall, "fits_per_s": len(cohorts) / con_wall,
            "same_tau": same,
            "config": "fit_null::run per cohort (counts, QC, GRM, AI-REML), .bed uploaded once; "
                      "concurrent: counts, QC and GRM rows of all cohorts under the streamed "
                      "upload, fits on a pool of host threads with their own streams; after one "
                      "untimed call of each mode, medians of three alternating runs"}
    # the reference's strategy on the same GPU
    plain_kv = None
    if not args.no_plain and world == 1:
        grm.precision = cs.PREC_FP32
        # FP32, one PCG per right-hand side, zero starts, the command's tolerance
        plain_cfg = cs.AiRemlConfig(tol=CLI_TOL, max_iter=30)
        t0 = time.perf_counter()
        pr = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, plain_cfg)
        pw = time.perf_counter() - t0
        solves = p + 2 + 30
        plain_kv = ref_kv_count(pr.iterations, p, 30, pr.pcg_iters, solves)
        line["plain"] = {"seconds": pr.seconds, "wall_s": pw, "pcg_iters": int(pr.pcg_iters),
                         "ai_reml_iterations": int(pr.iterations), "n_kv": int(pr.n_kv),
                         "reference_kv_per_fit": int(plain_kv),
                         "tau": [float(pr.tau[0]), float(pr.tau[1])]}
        line["speedup_vs_plain"] = pr.seconds / step_s
        line["tau_rel_diff_vs_plain"] = abs(float(last.tau[1]) - float(pr.tau[1])) / abs(float(pr.tau[1]))
        pd = cs.fit_ai_reml(y, x, grm, cs.TraitType.Binary, cs.AiRemlConfig())
        line["plain"]["default_tol"] = {
            "tol": 0.02, "seconds": pd.seconds, "pcg_iters": int(pd.pcg_iters),
            "ai_reml_iterations": int(pd.iterations), "n_kv": int(pd.n_kv),
            "reference_kv_per_fit": int(ref_kv_count(pd.iterations, p, 30, pd.pcg_iters, solves)),
            "tau": [float(pd.tau[0]), float(pd.tau[1])]}
        grm.precision = cs.PREC_MIXED
    # CPU baseline (rank 0): bounded sample, extrapolated with the reference product count
    if rank == 0 and world == 1:
        kv_fit = plain_kv or REF_KV_PER_FIT
        smp = CpuSample(n, min(CPU_SAMPLE_MARKERS, m))
        times = [smp.product_seconds() for _ in range(3)]
        per_kv = statistics.median(times) * m / smp.markers
        line["cpu_baseline"] = {
            "value": per_kv * kv_fit, "unit": "s", "cores": smp.threads, "kind": "port",
            "sample": smp.describe(m, kv_fit), "extrapolated": True, "sec_per_kv": per_kv}
        # the same per-product CPU time, times each extra path's reference product count
        if "variance_ratio" in line:
            vr = line["variance_ratio"]
            vr["cpu_extrapolated_s"] = per_kv * vr["reference_kv_estimate"]
            vr["cpu_note"] = ("reference products (one PCG per used marker) x the CPU port's "
                              "seconds per product")
        if "loco" in line and loco_sizes is not None:
            mg = float(sum(loco_sizes))
            line["loco"]["cpu_extrapolated_s"] = sum(per_kv * kv_fit * (mg - mc) / mg
                                                     for mc in loco_sizes)
            line["loco"]["cpu_note"] = ("22 fits x the reference strategy's product count x the "
                                        "CPU port's seconds per product, scaled by M - M_chrom")
    if rank == 0 and world == 1 and not args.no_config1:
        line["config1"] = config1_block(cs)
    if rank == 0 and world == 1 and not args.no_accuracy:
        del grm
        line["accuracy"] = accuracy_block(cs)
    if rank == 0 and world == 1 and not args.no_plain_scale:
        try:
            line["plain_gpu_scale"] = plain_scale_block(cs)
        except Exception as e:  # a side block: its failure must not cost the bench line
            line["plain_gpu_scale"] = {"error": repr(e)[:300]}
    if rank == 0 and world == 1 and not args.no_learned:
        line["config5_starts"] = starts_block(cs)
    if rank == 0 and world == 1 and not args.no_explicit_grm:
        line["explicit_grm"] = explicit_grm_block(cs, local, args.grm_n, args.grm_m,
                                                  args.grm_reps)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.explicit_grm_only:
        if rank == 0:
            import torch

            import csaige_b200 as cs
            torch.cuda.set_device(local)
            print(json.dumps(explicit_grm_block(cs, local, args.grm_n, args.grm_m, args.grm_reps,
                                                cpu=False)), flush=True)
        return
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
