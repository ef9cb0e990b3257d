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
REF_KV_PER_FIT = None  # filled in from a measured plain fit when available

FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-strategy fit")
    ap.add_argument("--no-e2e", action="store_true")
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def ref_kv_count(iterations: int, p: int, nrv: int, pcg_iters: int, solves_per_iter: int) -> int:
    """GRM products of the reference strategy: PCG iterations, one A*0 product
    per solve, and K*Py plus the probe products every iteration."""
    return pcg_iters + iterations * solves_per_iter + iterations * (1 + nrv)


# ---------------------------------------------------------------------------
# reference arm: CPU restatement, bounded marker sample, extrapolated
# ---------------------------------------------------------------------------
def cpu_kv_seconds(n: int, m_full: int, sample_markers: int, reps: int):
    sys.path.insert(0, str(ROOT / "tests"))
    import numpy as np

    import csaige_b200 as cs
    import oracle_ffi as O

    O.L.orc_grm_matvec_f32_packed.restype = C.c_int
    O.L.orc_grm_matvec_f32_packed.argtypes = [C.POINTER(C.c_uint8), C.c_int64, C.c_int64,
                                              C.POINTER(C.c_int64), C.c_int64, O._d, O._d, O._d,
                                              C.c_int]
    spec = cs.CohortSpec(n=n, m=sample_markers, seed=WORKLOAD["seed"],
                         sib_frac=WORKLOAD["sib_frac"], cousin_frac=WORKLOAD["cousin_frac"],
                         missing_rate=WORKLOAD["missing_rate"])
    bed = cs.gen_bed(spec)
    af, _, _ = O.marker_stats(bed, n, sample_markers)
    body = np.ascontiguousarray(bed[3:])
    rows = np.arange(sample_markers, dtype=np.int64)
    v = np.random.default_rng(1).standard_normal(n)
    out = np.empty(n)
    bpm = (n + 3) // 4
    times = []
    threads = 0
    for _ in range(reps):
        t0 = time.perf_counter()
        threads = O.L.orc_grm_matvec_f32_packed(body.ctypes.data_as(C.POINTER(C.c_uint8)), bpm, n,
                                                rows.ctypes.data_as(C.POINTER(C.c_int64)),
                                                sample_markers, O.dp(af), O.dp(v), O.dp(out), 0)
        times.append(time.perf_counter() - t0)
    per_kv = statistics.median(times) * m_full / sample_markers
    return per_kv, threads, times


def run_reference(args, rank):
    if rank != 0:
        return
    steps = []
    sample = 2048
    per_kv = threads = None
    kv_fit = _plain_kv_estimate()
    for _ in range(args.warmup + args.steps):
        per_kv, threads, _ = cpu_kv_seconds(args.n, args.m, sample, 1)
        steps.append(per_kv * kv_fit)
    timed = steps[args.warmup:]
    val = statistics.median(timed)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": val * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": _config(args),
        "cpu_baseline": {"value": val, "unit": "s", "cores": threads, "kind": "port",
                         "sample": f"OnTheFlyGrm::mat_vec arithmetic on {sample} of {args.m} "
                                   f"markers x {args.n} samples, x{args.m / sample:.1f} per "
                                   f"product, x{kv_fit} products per fit",
                         "sec_per_kv": per_kv},
        "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _plain_kv_estimate() -> int:
    """GRM products of one reference-strategy fit on this workload (see
    profiles/plain_fit_n200k_m150k.txt); 0 when unknown."""
    p = ROOT / "profiles" / "plain_fit_n200k_m150k.txt"
    if p.exists():
        for ln in p.read_text().splitlines():
            if ln.startswith("reference_kv_per_fit"):
                return int(ln.split("=")[1])
    return 0


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

    fast = cs.AiRemlConfig(precision=cs.PREC_MIXED, solve=cs.SOLVE_BLOCK,
                           warm_start=cs.WARM_PREVIOUS)
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
    step_s = statistics.mean(dev_s)
    if world > 1:
        t = torch.tensor([step_s], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        step_s = float(t.item())
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
    cols = st["n_kv"] / max(st["tc_pass_a_launches"], 1)  # right-hand sides per launch
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
    roof["traffic"] = None
    roof["kernel"] = f"tc_grm_kernel pass {dom} (MIXED, {cols:.1f} rhs per launch)"
    roof["peak_source"] = (f"{pk_kind} MEASURED_PEAKS.json" if pk_kind == "measured" else "fallback")
    roof["avg_launch_ms"] = avg_s * 1e3
    roof["share_of_step"] = (st["tc_pass_a_ms"] + st["tc_pass_b_ms"]) / 1e3 / (step_s * args.steps)

    line = {
        "metric": METRIC, "value": step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8 tensor products, f64 solver",
        "data": "synthetic", "config": _config(args),
        "pcg_iters": int(last.pcg_iters), "ai_reml_iterations": int(last.iterations),
        "tau": [float(last.tau[0]), float(last.tau[1])], "n_kv": int(last.n_kv),
        "n_kv_launches": int(last.n_kv_launches), "wall_s_per_step": wall / args.steps,
        "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary(),
        "markers_grm": int(m_grm), "markers_vr": int(len(vidx)),
        "fast_config": "MIXED + block PCG + previous-iterate warm start",
    }

    # end to end through the host-buffer C ABI
    if host_bed is not None:
        hb = host_bed.numpy()
        cs.fit_null_from_bed(hb, n, m, y, x, cs.TraitType.Binary, fast)  # warm-up
        e2e_t = []
        for _ in range(min(args.steps, 2)):
            t0 = time.perf_counter()
            fr = cs.fit_null_from_bed(hb, n, m, y, x, cs.TraitType.Binary, fast)
            e2e_t.append(time.perf_counter() - t0)
        line["e2e"] = {"value": statistics.mean(e2e_t), "unit": "s",
                       "h2d_bytes_per_step": int(spec.bed_len + y.nbytes + x.nbytes),
                       "d2h_bytes_per_step": int(8 * (p + n + 2 * fast.max_iter)),
                       "tau": [float(fr.ai_reml.tau[0]), float(fr.ai_reml.tau[1])]}
    # the reference's strategy on the same GPU
    plain_kv = None
    if not args.no_plain and world == 1:
        grm.precision = cs.PREC_FP32
        plain_cfg = cs.AiRemlConfig()  # FP32, one PCG per right-hand side, zero starts
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
    # CPU baseline (rank 0): bounded sample, extrapolated with the reference product count
    if rank == 0 and world == 1:
        kv_fit = plain_kv or _plain_kv_estimate()
        if kv_fit:
            per_kv, threads, times = cpu_kv_seconds(n, m, 2048, 3)
            line["cpu_baseline"] = {
                "value": per_kv * kv_fit, "unit": "s", "cores": threads, "kind": "port",
                "sample": f"OnTheFlyGrm::mat_vec arithmetic (f32, per-thread fold) on 2048 of {m} "
                          f"markers x {n} samples, extrapolated x{m / 2048:.1f} per product and "
                          f"x{kv_fit} products per fit (reference strategy count)",
                "sec_per_kv": per_kv}
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
    run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
