#!/usr/bin/env python
"""k-NN benchmark: queries/second on one or more B200s, one JSON line.

Workload (default ``mixture256``): ref_nb = 1,048,576 reference points,
query_nb = 16,384 queries, dim = 256, k = 100, a seeded Gaussian mixture of
1024 unit-norm centres (sigma 0.1).  A "step" is one k-NN pass of the query
batch over the whole reference set.  Inputs are larger than L2 (the
reference set alone is 1 GiB), so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* ``--impl ours`` (default) measures both tiers of the metric on the
  device-resident entry point (inputs already in HBM, CUDA events on the
  launching stream, max over ranks): ``exact_fp32`` (the fused direct-form
  kernel behind knn_cuda_global) and ``bf16_rerank`` (tcgen05 BF16 scan +
  exact FP32 re-rank behind knn_cublas; its answers are checked identical to
  the exact tier's and against an FP64 brute force on sampled queries).
  ``value`` is the bf16_rerank tier; ``e2e`` is the same metric through the
  drop-in host entry point knn_cublas with pinned host buffers, every
  host<->device copy inside the timed region.  ``roofline`` reports the
  pass-2 tensor scan (per-kernel CUDA events inside the library) against the
  measured bf16 peak; the exact tier carries its own FP32 roofline against
  the FP32 FMA throughput measured in the same run.  ``cpu_baseline`` = the
  reference's own knn_c on the host cores (rank 0).
* ``--impl reference``: the reference's own CPU implementation (knn_c,
  code/test.cpp:129-175, built from its sources into oracle/_ref) on all
  host threads, each step a bounded sample of queries over the full
  reference set.

Multi-GPU: one process per GPU (torchrun); every rank runs its own query
batch against a replica of the reference set (queries are independent, no
data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "knn-cuda_b200")
for _p in (PKG, ROOT):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import workloads  # noqa: E402

METRIC = "kNN queries/sec (N=1M,d=256,k=100): FP32 exact vs BF16+rerank @ recall=1.0"
UNIT = "queries/s"

# DRAM traffic (read + write bytes) per launch of the dominant kernel, from
# the ncu capture summarised in profiles/, keyed by (kernel, workload,
# queries), with the source it was captured at; None for a configuration
# that was not captured.  A capture is not repeated by this script: after a
# change to the kernel the entry is stale until it is captured again.
NCU_TRAFFIC = {
    ("knn_tc_pair_scan_kernel<1>", "mixture256", 16384): {
        # dram__bytes_read.sum 655,172,352 + dram__bytes_write.sum 42,589,696
        "bytes": 655172352 + 42589696,
        "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one pass-2 launch, "
                  "16384 queries, 23 splits (profiles/knn_tc_pair_scan_pass2_mixture256.md)",
    },
}


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", default="mixture256", choices=sorted(workloads.WORKLOADS))
    p.add_argument("--queries", type=int, default=0, help="override query_nb per rank")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="target CPU time of the bounded knn_c sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp8-forced", action="store_true",
                   help="skip the measurement of an FP8 pass 2 forced on the workload")
    p.add_argument("--mode", choices=["batch", "serving", "batched"], default="batch",
                   help="serving: resident serving128 set, Poisson request stream; "
                        "batched: 512 uneven problems, one persistent launch vs per-problem")
    p.add_argument("--serve-seconds", type=float, default=20.0)
    p.add_argument("--ref-gpu", choices=["", "cublas", "global"], default="",
                   help="with --impl reference: time the reference's own GPU function "
                        "(built from its sources) instead of its CPU knn_c")
    p.add_argument("--ref-chunks", type=int, default=2,
                   help="query chunks of 1024 timed for --ref-gpu")
    return p.parse_args(argv)


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend="nccl"):
        import torch

        if torch.cuda.is_available():
            torch.cuda.set_device(self.local_rank)
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch
            import torch.distributed as dist

            dist.barrier(device_ids=[self.local_rank] if torch.cuda.is_available() else None)

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist

        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{self.local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            import torch.distributed as dist

            dist.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        load = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own knn_c (oracle/_ref), all host threads
# ---------------------------------------------------------------------------
def cpu_sample_rate(ref, query, k, seconds_target: float, max_rounds: int = 1):
    """Time the reference knn_c on a bounded query sample; returns
    (queries/s, threads, sample description, kind)."""
    from oracle import oracle

    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    fn = oracle.ref_knn_c if kind == "reference" else oracle.knn_c
    # calibrate with one query per thread
    qn = min(threads, query.shape[1])
    t0 = time.perf_counter()
    fn(ref, np.ascontiguousarray(query[:, :qn]), k, threads=threads)
    t1 = time.perf_counter() - t0
    per_round = max(qn, int(qn * max(1.0, seconds_target / max(t1, 1e-3))))
    per_round = min(per_round, query.shape[1])
    rates = []
    for _ in range(max_rounds):
        t0 = time.perf_counter()
        out = fn(ref, np.ascontiguousarray(query[:, :per_round]), k, threads=threads)
        rates.append(per_round / (time.perf_counter() - t0))
    desc = (f"first {per_round} queries of the workload against all {ref.shape[1]} reference "
            f"points, {threads} threads over contiguous query slices; per-query cost is "
            f"independent of the other queries, so queries/s scales to the full batch")
    return rates, threads, desc, kind, per_round, out


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            m = json.load(f)
        return {"bf16_tflops": float(m["bf16_tflops"]), "hbm_gbs": float(m["hbm_gbs"]),
                "source": "measured (MEASURED_PEAKS.json, burst)"}
    except (OSError, KeyError, ValueError):
        return {"bf16_tflops": 1590.0, "hbm_gbs": 6650.0, "source": "fallback"}


def time_tier(knncuda, torch, D, stream, step, steps, clocks=None):
    """Run `steps` timed steps; per-step sync to read the library's phase
    timers.  Returns (ms per step, max over ranks; mean phase ms)."""
    D.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    knncuda.set_phase_timing(True)
    phase_sum, second, exact, cands = {}, 0, 0, 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
        torch.cuda.synchronize()
        for k, v in knncuda.last_phase_times().items():
            phase_sum[k] = phase_sum.get(k, 0.0) + v
        st = knncuda.last_tc_stats()
        second, exact = second + st["second_scan"], exact + st["exact"]
        cands += st["candidates"]
    e1.record(stream)
    torch.cuda.synchronize()
    knncuda.set_phase_timing(False)
    D.barrier()
    clk = clocks.stop() if clocks else None
    if knncuda.sync_status() != 0:
        raise RuntimeError("device status error in timed region")
    ms = D.max(e0.elapsed_time(e1) / steps)
    return (ms, {k: v / steps for k, v in phase_sum.items()},
            {"second_scan": second / steps, "exact": exact / steps,
             "candidates": cands / steps}, clk)


def fp64_recall(torch, ref_d, qry_d, idx, dist, k, sample):
    """recall@k and max relative distance error of sampled queries against an
    FP64 brute force computed on the GPU."""
    r64 = ref_d.double()
    hits, worst = 0, 0.0
    for q in sample:
        q64 = qry_d[:, q].double()
        d2 = ((r64 - q64[:, None]) ** 2).sum(0)
        top = torch.topk(d2, k, largest=False)
        truth = set(top.indices.tolist())
        mine = idx[:, q].long()
        hits += len(truth & set(mine.tolist()))
        exact = torch.sqrt(d2[mine])
        rel = ((dist[:, q].double() - exact).abs() / exact.clamp_min(1e-12)).max().item()
        worst = max(worst, rel)
    return hits / (k * len(sample)), worst


def fp8_forced(knncuda, torch, dev, ref_d, qry_d, k, stream, outs, steps=2):
    """The FP8 request with pass 2 forced to FP8 (the library's test and
    measurement override), timed like the tiers: what an FP8 candidate scan
    costs on this data, answers still exact."""
    qn = qry_d.shape[1]
    d = torch.empty((k, qn), dtype=torch.float32, device=dev)
    i = torch.empty((k, qn), dtype=torch.int32, device=dev)
    knncuda.set_tc_kind_override("fp8")
    try:
        knncuda.knn_device(ref_d, qry_d, k, "fp8", d, i, stream)
        torch.cuda.synchronize(dev)
        knncuda.set_phase_timing(True)
        ph, st = {}, {}
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            knncuda.knn_device(ref_d, qry_d, k, "fp8", d, i, stream)
            torch.cuda.synchronize(dev)
            for kk, v in knncuda.last_phase_times().items():
                ph[kk] = ph.get(kk, 0.0) + v / steps
            st = knncuda.last_tc_stats()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        knncuda.set_phase_timing(False)
        kinds = knncuda.last_tc_kinds()
    finally:
        knncuda.set_tc_kind_override(None)
    ms = e0.elapsed_time(e1) / steps
    return {"value": qn / (ms * 1e-3), "ms_per_step": ms,
            "phase_ms": {kk: round(v, 4) for kk, v in ph.items()},
            "scan_kinds": {"pass2": kinds[0], "second_scan": kinds[1]},
            "first_scan_candidates": st.get("candidates"),
            "second_scan_queries": st.get("second_scan"), "exact_queries": st.get("exact"),
            "identical_to_exact": bool(torch.equal(d, outs["exact_fp32"][0]) and
                                       torch.equal(i, outs["exact_fp32"][1]))}


def run_ours(args, D: Dist):
    import torch

    import knncuda

    D.init("nccl")
    dev = torch.device(f"cuda:{D.local_rank}")
    w = workloads.WORKLOADS[args.workload]
    qn = args.queries or w.query_nb
    ref, query = workloads.generate(w, query_nb=qn)
    dim, N = ref.shape
    k = w.k
    # pinned host copies (e2e) and device-resident copies (value)
    ref_h = torch.from_numpy(ref).pin_memory()
    qry_h = torch.from_numpy(query).pin_memory()
    ref_d = ref_h.to(dev)
    qry_d = qry_h.to(dev)
    stream = torch.cuda.current_stream(dev)
    peaks = measured_peaks()
    warm = max(3, args.warmup)
    tiers = {}
    outs = {}
    tier_methods = [("exact_fp32", "global"), ("bf16_rerank", "cublas"), ("fp8_rerank", "fp8")]
    for name, method in tier_methods:
        dist_d = torch.empty((k, qn), dtype=torch.float32, device=dev)
        idx_d = torch.empty((k, qn), dtype=torch.int32, device=dev)

        def step(method=method, dist_d=dist_d, idx_d=idx_d):
            knncuda.knn_device(ref_d, qry_d, k, method, dist_d, idx_d, stream)

        for _ in range(warm):
            step()
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(D.local_rank) if name == "bf16_rerank" else None
        ms, phases, fb, clk = time_tier(knncuda, torch, D, stream, step, args.steps, clocks)
        outs[name] = (dist_d, idx_d)
        tiers[name] = {"value": D.world * qn / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                       "phase_ms": phases, "uncertified_queries_per_step": fb}
        if method != "global":
            first, second = knncuda.last_tc_kinds()
            tiers[name]["scan_kinds"] = {"pass2": first, "second_scan": second}
        if clk is not None:
            tiers[name]["clocks"] = clk

    # identical answers, and recall / error against FP64 on sampled queries
    sample = list(range(0, qn, max(1, qn // 32)))[:32]
    for name, _ in tier_methods:
        same = bool(torch.equal(outs["exact_fp32"][0], outs[name][0]) and
                    torch.equal(outs["exact_fp32"][1], outs[name][1]))
        recall, relerr = fp64_recall(torch, ref_d, qry_d, outs[name][1], outs[name][0], k,
                                     sample)
        tiers[name].update(identical_to_exact=same, recall_at_k_fp64=recall,
                           max_rel_dist_err_fp64=relerr, fp64_sample_queries=len(sample))
    f8 = tiers["fp8_rerank"]
    f8["vs_bf16_rerank"] = f8["value"] / tiers["bf16_rerank"]["value"]
    if f8.get("scan_kinds", {}).get("pass2") != "fp8":
        f8["note"] = ("the BF16 sample pass predicted overflowing FP8 candidate lists (the FP8 "
                      "error bound exceeds this data's distance spread): pass 2 ran in BF16; "
                      "fp8_forced is the same call with pass 2 forced to FP8")
    if not args.no_fp8_forced:
        f8["fp8_forced"] = fp8_forced(knncuda, torch, dev, ref_d, qry_d, k, stream, outs)

    # end to end through the drop-in host entry points (pinned buffers)
    ref_np, qry_np = ref_h.numpy(), qry_h.numpy()
    out_d = torch.empty((k, qn), dtype=torch.float32).pin_memory().numpy()
    out_i = torch.empty((k, qn), dtype=torch.int32).pin_memory().numpy()
    e2e = {}
    # the reference's harness passes malloc'd (pageable) buffers
    # (code/test.cpp:314-317): knn_cublas from pageable memory
    out_pd = np.empty((k, qn), np.float32)
    out_pi = np.empty((k, qn), np.int32)
    ref_pg, qry_pg = np.array(ref_np), np.array(qry_np)
    knncuda.knn_cublas(ref_pg, N, qry_pg, qn, dim, k, out_pd, out_pi)
    D.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        if not knncuda.knn_cublas(ref_pg, N, qry_pg, qn, dim, k, out_pd, out_pi):
            raise RuntimeError("knn_cublas (pageable) failed")
    e2e_pageable = D.max((time.perf_counter() - t0) / args.e2e_steps)
    if not np.array_equal(out_pi, outs["exact_fp32"][1].cpu().numpy()):
        raise RuntimeError("pageable knn_cublas disagrees with the device path")
    for name, fn in (("exact_fp32", knncuda.knn_cuda_global),
                     ("bf16_rerank", knncuda.knn_cublas)):
        fn(ref_np, N, qry_np, qn, dim, k, out_d, out_i)   # warm (workspace growth)
        D.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            if not fn(ref_np, N, qry_np, qn, dim, k, out_d, out_i):
                raise RuntimeError(f"{name} host entry failed")
        e2e[name] = D.max((time.perf_counter() - t0) / args.e2e_steps)
        if not (np.array_equal(out_i, outs["exact_fp32"][1].cpu().numpy()) and
                np.array_equal(out_d, outs["exact_fp32"][0].cpu().numpy())):
            raise RuntimeError(f"host entry {name} disagrees with the device path")
        tiers[name]["e2e_value"] = D.world * qn / e2e[name]

    head = tiers["bf16_rerank"]
    tensor_path = "tc_pass2" in head["phase_ms"]
    ref_mb = ref.nbytes / 2**20
    l2_note = (f"inputs larger than L2 ({ref_mb:.0f} MiB reference set); no flush"
               if ref.nbytes > 126 * 2**20 else
               f"the {ref_mb:.0f} MiB reference set fits in L2 and is not flushed between "
               "steps (warm-L2 figure)")
    d_pad = (dim + 63) // 64 * 64
    pass2_ms = head["phase_ms"].get("tc_pass2")
    flops = 2.0 * d_pad * N * qn
    achieved = flops / (pass2_ms * 1e-3) if pass2_ms else None
    peak = peaks["bf16_tflops"] * 1e12
    fb = head["uncertified_queries_per_step"]
    # reference prep 3 (center, prep, sample rows) + query prep 2 + pass 1 +
    # threshold + pass 2 + re-rank 3 (select, gather, certify); second scan
    # 7 more; exact fallback 5 more (gather, query copy, fused kernel, split
    # merge, scatter)
    launches = 11 + (7 if fb["second_scan"] > 0 else 0) + (5 if fb["exact"] > 0 else 0)
    ex = tiers["exact_fp32"]
    ex_ms = ex["phase_ms"].get("exact_main", ex["ms_per_step"])
    fp32_peak = knncuda.measure_fp32_peak(8192)
    ex["roofline"] = {"bound": "fp32", "kernel": "knn_exact_kernel<4,128> (fused exact FP32)",
                      "achieved": 3.0 * dim * N * qn / (ex_ms * 1e-3) / 1e12,
                      "peak": fp32_peak / 1e12, "unit": "TFLOP/s",
                      "frac": 3.0 * dim * N * qn / (ex_ms * 1e-3) / fp32_peak,
                      "algorithmic": "3*dim flops per (query, reference) pair",
                      "peak_source": "FP32 FMA throughput measured in this run"}

    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": D.world,
        "steps": args.steps, "warmup": warm, "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16" if tensor_path else "f32",
        "data": w.data_text(),
        "impl": "ours",
        "config": dict(w.describe(), query_nb=qn,
                       tier=("bf16_rerank: tcgen05 BF16 scan + exact FP32 re-rank (knn_cublas)"
                             if tensor_path else
                             "bf16_rerank tier (knn_cublas): this shape runs the exact FP32 "
                             "kernels (tensor path needs 16 <= dim and ref_nb >= 32768)"),
                       parallelism=f"query-sharded replicas x{D.world}",
                       l2=l2_note),
        "e2e": {"value": D.world * qn / e2e["bf16_rerank"], "unit": UNIT,
                "h2d_bytes_per_step": int(ref.nbytes + query.nbytes),
                "d2h_bytes_per_step": int(out_d.nbytes + out_i.nbytes),
                "api": "knn_cublas (drop-in C-ABI, pinned host buffers)",
                "ms_per_step": e2e["bf16_rerank"] * 1e3},
        "gpu_launches": launches * args.steps,
        "roofline": {"bound": "tensor",
                     "kernel": "knn_tc_pair_scan_kernel<1> (pass-2 scan on CTA pairs)",
                     "achieved": achieved / 1e12 if achieved else None,
                     "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                     "frac": achieved / peak if achieved else None,
                     "traffic": (NCU_TRAFFIC.get(("knn_tc_pair_scan_kernel<1>", w.name, qn))
                                 or {}).get("bytes"),
                     "traffic_source": (NCU_TRAFFIC.get(
                         ("knn_tc_pair_scan_kernel<1>", w.name, qn)) or {}).get("source"),
                     "algorithmic": f"2*d_pad flops per (query, reference) pair, d_pad={d_pad}"
                                    + (" (split BF16 issues 3 MMAs per K step: 3x this work on "
                                       "the tensor pipe)" if head.get("scan_kinds", {}).get("pass2")
                                       == "bf16x3" else ""),
                     "peak_source": peaks["source"]},
        "clocks": head.get("clocks"),
        "tiers": tiers,
        "speedup_bf16_vs_exact": head["value"] / ex["value"],
        "e2e_pageable": {"value": D.world * qn / e2e_pageable, "unit": UNIT,
                         "ms_per_step": e2e_pageable * 1e3,
                         "api": "knn_cublas (drop-in C-ABI, pageable numpy buffers as in "
                                "code/test.cpp)"},
    }
    if D.rank == 0 and D.world == 1 and not args.no_cpu_baseline:
        rates, threads, desc, kind, qs, (gt_d, gt_i) = cpu_sample_rate(ref, query, k,
                                                                        args.cpu_seconds)
        line["cpu_baseline"] = {"value": rates[0], "unit": UNIT, "cores": threads,
                                "kind": kind, "sample": desc}
        # the reference harness's pass rule (code/test.cpp:216-217, :256-272)
        # on the sampled queries, against the knn_c outputs just timed
        from oracle import oracle
        for name, (dd, ii) in outs.items():
            od = dd[:, :qs].cpu().numpy()
            oi = ii[:, :qs].cpu().numpy()
            ok, dacc, iacc = oracle.reference_criterion(od, oi, gt_d, gt_i)
            tiers[name]["knn_c_criterion"] = {
                "queries": int(qs), "passed": bool(ok), "dist_acc": dacc, "index_acc": iacc,
                "max_abs_dist_diff": float(np.max(np.abs(od.astype(np.float64) - gt_d)))}
    if D.rank == 0:
        print(json.dumps(line), flush=True)
    D.close()


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU implementation on all host threads
# ---------------------------------------------------------------------------
def run_reference_gpu(args, D: Dist):
    """The reference's own GPU knn_cublas / knn_cuda_global (code/knncuda.cu,
    built unmodified into oracle/_ref/libknnref_gpu.so), called through its
    host API, inside its limits: ref_nb <= 1,048,560 (grid-y) and a multiple
    of 128 (knn_cublas needs ref_pitch == ref_nb), queries in chunks of 1024
    so ref_nb * query_pitch < 2^31 (32-bit index math)."""
    import ctypes

    from oracle import oracle

    w = workloads.WORKLOADS[args.workload]
    ref, query = workloads.generate(w)
    dim, N = ref.shape
    n_ref = min(N, 1048560) // 128 * 128
    ref = np.ascontiguousarray(ref[:, :n_ref])
    chunk = min(1024, query.shape[1])
    lib = ctypes.CDLL(oracle.REF_GPU_SO)
    names = {"cublas": "_Z10knn_cublasPKfiS0_iiiPfPi",
             "global": "_Z15knn_cuda_globalPKfiS0_iiiPfPi"}
    fn = getattr(lib, names[args.ref_gpu])
    fp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
    fn.restype = ctypes.c_bool
    fn.argtypes = [fp, ctypes.c_int, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, fp, ip]
    k = w.k
    dist = np.empty((k, chunk), np.float32)
    idx = np.empty((k, chunk), np.int32)
    qs = [np.ascontiguousarray(query[:, i * chunk:(i + 1) * chunk]) for i in range(args.ref_chunks + 1)]
    call = lambda q: fn(ref.ctypes.data_as(fp), n_ref, q.ctypes.data_as(fp), chunk, dim, k,
                        dist.ctypes.data_as(fp), idx.ctypes.data_as(ip))
    if not call(qs[0]):
        raise RuntimeError("reference GPU function failed")
    t0 = time.perf_counter()
    for q in qs[1:args.ref_chunks + 1]:
        if not call(q):
            raise RuntimeError("reference GPU function failed")
    s = (time.perf_counter() - t0) / args.ref_chunks
    value = chunk / s
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.ref_chunks,
        "warmup": 1, "ms_per_step": s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
        "reference_path": f"knn_{'cublas' if args.ref_gpu == 'cublas' else 'cuda_global'} "
                          "(reference GPU code, host API, per-call alloc + H2D + D2H)",
        "config": dict(w.describe(), ref_nb_used=n_ref, query_chunk=chunk,
                       note="ref_nb trimmed to the reference's limits; per-query cost "
                            "scales ~linearly with ref_nb"),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(ref.nbytes + qs[0].nbytes),
                "d2h_bytes_per_step": int(dist.nbytes + idx.nbytes)}}), flush=True)


def run_reference(args, D: Dist):
    if D.rank != 0:
        return
    if args.ref_gpu:
        return run_reference_gpu(args, D)
    from oracle import oracle

    w = workloads.WORKLOADS[args.workload]
    qn = args.queries or w.query_nb
    ref, query = workloads.generate(w, query_nb=qn)
    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    fn = oracle.ref_knn_c if kind == "reference" else oracle.knn_c
    # each step: a bounded sample of queries sized to about cpu_seconds / 3
    qs = min(threads, qn)
    t0 = time.perf_counter()
    fn(ref, np.ascontiguousarray(query[:, :qs]), w.k, threads=threads)
    t1 = time.perf_counter() - t0
    per_step = min(qn, max(qs, int(qs * max(1.0, (args.cpu_seconds / 3) / max(t1, 1e-3)))))
    sample = np.ascontiguousarray(query[:, :per_step])
    for _ in range(args.warmup):
        fn(ref, sample, w.k, threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        fn(ref, sample, w.k, threads=threads)
        times.append(time.perf_counter() - t0)
    s = sum(times) / len(times)
    value = per_step / s
    desc = (f"{per_step} queries per step against all {ref.shape[1]} reference points, "
            f"{threads} threads over contiguous query slices (reference knn_c, "
            f"code/test.cpp:129-175)")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": D.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "impl": "reference",
        "config": dict(w.describe(), query_nb=qn, sample_queries_per_step=per_step),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
# serving: resident reference set, Poisson request stream, continuous batching
# ---------------------------------------------------------------------------
def run_serving(args, D: Dist):
    import random
    import threading

    import torch

    import knncuda

    D.init("nccl")
    w = workloads.WORKLOADS["serving128"]
    ref, _ = workloads.generate(w, query_nb=1)
    rs = knncuda.RefSet(ref)
    reqs = workloads.serving_requests(w, 4000)

    def drive(rate_hz, seconds, method, window=0):
        """window > 0: closed loop with `window` requests outstanding;
        otherwise open loop with Poisson arrivals at rate_hz."""
        import collections

        srv = knncuda.Server(rs, slots=3, memory_budget=16 << 30, max_batch_queries=8192,
                             method=method)
        pending = collections.deque()
        rnd = random.Random(7)
        i = 0
        t_end = time.perf_counter() + seconds
        t_next = time.perf_counter()
        while time.perf_counter() < t_end:
            if window:
                while len(pending) >= window:
                    srv.wait(pending.popleft())
            else:
                delay = t_next - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                t_next += rnd.expovariate(rate_hz)
                while len(pending) >= 4096:          # bound host memory if overloaded
                    srv.wait(pending.popleft())
            pending.append(srv.submit(*reqs[i % len(reqs)]))
            i += 1
        while pending:
            srv.wait(pending.popleft())
        st = srv.stats()
        srv.close()
        st["requests"] = i
        st["qps"] = st["queries"] / st["wall_s"] if st["wall_s"] > 0 else 0.0
        return st

    out = {}
    for method in ("cublas", "global"):
        drive(0, 1.0, method, window=8)            # warm the slots
        sat = drive(0, min(5.0, args.serve_seconds / 4), method, window=24)  # capacity
        mean_q = float(np.mean([q.shape[1] for q, _ in reqs]))
        rate = 0.7 * sat["qps"] / mean_q            # offered load: 70 % of capacity
        open_loop = drive(rate, args.serve_seconds, method)
        out[method] = {"saturation_qps": sat["qps"], "offered_requests_per_s": rate,
                       "qps": open_loop["qps"], "p50_ms": open_loop["p50_ms"],
                       "p99_ms": open_loop["p99_ms"], "requests": open_loop["requests"],
                       "batches": open_loop["batches"]}
    # exactness of served results: 16 requests against an FP64 brute force
    # on the GPU (first and last query of each)
    ref_d = torch.from_numpy(ref).to(torch.device(f"cuda:{D.local_rank}"))
    srv = knncuda.Server(rs, slots=3, memory_budget=16 << 30, max_batch_queries=8192,
                         method="cublas")
    chk = [reqs[j] for j in range(0, 16 * 7, 7)]
    tickets = [srv.submit(q, k) for q, k in chk]
    hits, total, worst = 0.0, 0, 0.0
    for (q, k), t in zip(chk, tickets):
        d, i, _ = srv.wait(t)
        qd = torch.from_numpy(q).to(ref_d.device)
        sample = sorted({0, q.shape[1] - 1})
        rec, err = fp64_recall(torch, ref_d, qd, torch.from_numpy(i).to(ref_d.device),
                               torch.from_numpy(d).to(ref_d.device), k, sample)
        hits += rec * len(sample)
        total += len(sample)
        worst = max(worst, err)
    srv.close()
    out["cublas"].update(recall_at_k_fp64=hits / total, max_rel_dist_err_fp64=worst,
                         fp64_sample_queries=total)
    line = {"metric": "serving queries/s and p50/p99 latency (resident 2M x 128, k in {10,50,100})",
            "value": out["cublas"]["qps"], "unit": "queries/s", "n_gpus": D.world,
            "higher_is_better": True, "impl": "ours", "mode": "serving",
            "config": dict(w.describe(), refset_bytes=rs.device_bytes(),
                           arrivals="Poisson at 70 % of the capacity measured with 24 "
                                    "requests outstanding",
                           request_queries="log-uniform 1..1024"),
            "methods": out}
    if D.rank == 0:
        print(json.dumps(line), flush=True)
    rs.close()
    D.close()


# ---------------------------------------------------------------------------
# batched: 512 uneven problems, per-problem launches vs one persistent launch
# ---------------------------------------------------------------------------
def run_batched(args, D: Dist):
    import torch

    import knncuda

    D.init("nccl")
    dev = torch.device(f"cuda:{D.local_rank}")
    shapes = workloads.batched_problems()
    probs, outs = [], []
    for n, q, d, k, seed in shapes:
        g = torch.Generator(device=dev).manual_seed(seed)
        ldr, ldq = (n + 3) // 4 * 4, (q + 3) // 4 * 4
        ref = torch.rand((d, ldr), generator=g, device=dev)[:, :n]
        qry = torch.rand((d, ldq), generator=g, device=dev)[:, :q]
        probs.append((ref, qry, k))
        outs.append((torch.empty((k, q), device=dev), torch.empty((k, q), dtype=torch.int32,
                                                                   device=dev)))
    stream = torch.cuda.current_stream(dev)
    pairs = sum(q * n for n, q, d, k, _ in shapes)

    def per_problem():
        for (ref, qry, k), (dd, ii) in zip(probs, outs):
            knncuda.knn_device(ref, qry, k, "global", dd, ii, stream)

    def timed(fn, reps):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    ms_single = timed(per_problem, args.steps)
    ref_out = [(d.clone(), i.clone()) for d, i in outs]
    arr = knncuda.problems_from([(r, q, k, d, i) for (r, q, k), (d, i) in zip(probs, outs)])
    # the work-item-size tuner alone as the baseline configuration
    best_stages, _ = knncuda.batched_autotune(arr)
    plan0 = knncuda.BatchedPlan(arr, item_stages=best_stages)
    ms_items_only = timed(plan0.run, args.steps)
    plan0.close()
    best, tuned_ms = knncuda.batched_autotune_config(arr)
    plan = knncuda.BatchedPlan(arr, config=best)
    ms_batched = timed(plan.run, args.steps)
    plan.capture_graph()
    ms_graph = timed(plan.replay, args.steps)
    same = all(torch.equal(d, a) and torch.equal(i, b) for (d, i), (a, b) in zip(outs, ref_out))
    # exactness against FP64: first and last query of every 8th problem
    hits, total, worst = 0.0, 0, 0.0
    for (ref, qry, k), (d, i) in list(zip(probs, outs))[::8]:
        sample = sorted({0, qry.shape[1] - 1})
        rec, err = fp64_recall(torch, ref, qry, i, d, k, sample)
        hits += rec * len(sample)
        total += len(sample)
        worst = max(worst, err)
    if plan.status() != 0:
        raise RuntimeError("device status error")
    line = {"metric": "batched k-NN: 512 uneven problems per step",
            "value": 1e3 / ms_graph, "unit": "steps/s (512 problems each)", "n_gpus": D.world,
            "higher_is_better": True, "impl": "ours", "mode": "batched",
            "config": {"workload": "batched512", "problems": len(shapes),
                       "pairs_per_step": pairs, "autotuned": plan.config(),
                       "work_items": plan.items()},
            "ms_per_problem_launches": ms_single, "ms_persistent_launch": ms_batched,
            "ms_item_size_tuned_only": ms_items_only,
            "item_size_tuned_only": {"item_stages": best_stages},
            "ms_graph_replay": ms_graph, "speedup_vs_per_problem": ms_single / ms_graph,
            "identical_to_per_problem": same, "recall_at_k_fp64": hits / total,
            "max_rel_dist_err_fp64": worst, "fp64_sample_queries": total}
    plan.close()
    if D.rank == 0:
        print(json.dumps(line), flush=True)
    D.close()


def main(argv=None):
    args = parse_args(argv)
    D = Dist()
    if args.impl == "reference":
        run_reference(args, D)
    elif args.mode == "serving":
        run_serving(args, D)
    elif args.mode == "batched":
        run_batched(args, D)
    else:
        run_ours(args, D)


if __name__ == "__main__":
    main()
