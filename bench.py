#!/usr/bin/env python3
"""Benchmark of the NRG iteration hot path on B200 (one JSON line on stdout).

Headline workload (metric: NRG runs/hour and p50/p99 latency, served vs
plain FP64): the served z-averaging stream of single-impurity Anderson runs
(QS symmetry, flat band, U = 0.2, Gamma = 0.02, Lambda = 2, Nmax = 40, FDM
A(omega) at T = 1e-6, 50 bins per decade; z = k/8 crossed with seeded
eps_d in [-0.2, 0]; Nkeep drawn from {200, 500, 1000, 2000}).  One step is
one wave of 32 requests (one z value, the 32 eps_d values); the default 4
steps serve the first 128 requests of the 256-run stream.

  value      runs/hour of the stream through the run server (libnrgb,
             continuous batching), all requests queued at t = 0 (capacity),
             on the server's clock: first submission to last completion
  e2e        the same stream on the client's clock, including reading every
             run's result files back; h2d/d2h bytes per step are the runs'
             host<->device copies of one wave
  latency_s  p50/p99 time-to-spectrum with Poisson arrivals at 85% of the
             measured capacity
  plain      the same requests one after another through nrgb_run, with one
             batched eigensolver call per step and with one call per block
             (the reference's per-subspace dsyev structure), sampled per Nkeep
  split8     the same stream again with the products of the recalculations
             and density matrices in split precision (gemm_slices=8: INT8
             slices on the tensor cores), all queued at t = 0, with the
             largest per-bin relative difference of its spectra from the
             FP64 pass (bins above 1e-6 of each spectrum's largest)
  microbench the batched eigensolve + recalc step of 40 dense blocks of size
             16..4096 (log-uniform), batched against per-block solver calls,
             with the panel kernel's roofline
  --impl reference
             the reference's CPU algorithm (the oracle) on the host cores on a
             bounded sample of the same stream.

Multi-GPU (torchrun): runs do not shard; every rank serves its own copy of
the stream on its GPU (replicas, weak scaling); value is the sum over ranks
with the span taken as the max over ranks.
"""
from __future__ import annotations

import argparse
import copy
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nrgljubljana-old_b200"))

METRIC = "NRG runs/hour and p50/p99 latency, served vs plain FP64 (spectra <=1e-8 rel err)"
WAVE = 32           # requests per step (one z value x 32 eps_d)
LOAD = 0.85         # Poisson rate for the latency pass, as a fraction of capacity
LOAD_LOW = 0.5      # second latency pass, well below capacity
LAT_RUNS = 64       # requests in the latency pass
MAX_RUNS = 16       # worker slots of the server: 12..32 measured 16.7k-35.7k runs/hour on shared boxes, host load dominating

# microbenchmark: 40 dense blocks per step, 6 operators per block pair
NBLOCKS = 40
NOPS_PER_PAIR = 6
SEED = 20261204
NMAX = 4096


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap", "utilization.gpu"]

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == len(self.FIELDS):
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[0]) for r in self.rows) if v is not None]
        mx = [v for v in (num(r[1]) for r in self.rows) if v is not None]
        util = [v for v in (num(r[6]) for r in self.rows) if v is not None]
        reasons = set()
        for r in self.rows:
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], r[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "gpu_util_pct_median": statistics.median(util) if util else None}


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def fp64_gemm_peak(torch, dev):
    """Measured FP64 tensor GEMM throughput (cuBLAS DGEMM 8192^3, best of 5)."""
    n = 8192
    a = torch.randn(n, n, device=dev, dtype=torch.float64)
    b = torch.randn(n, n, device=dev, dtype=torch.float64)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1000.0)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


KERNELS = ("trd_panel", "trd_cluster", "gemm_f64_trailing", "gemm_f64_dc", "gemm_f64_bt", "gemm_f64_recalc", "gemm_f64_nrg",
           "dc_prep", "dc_permute", "dc_secular", "dc_lowner", "dc_vectors", "dc_rank", "dc_copy", "dc_leaf",
           "bt_T", "bt_buildV", "syev_small", "assemble*", "spec_dmnrg", "spec_fdm", "merge_bins",
           "gather_diag", "col_scale")


def kernel_table(ctx):
    return {k.rstrip("*"): ctx.kernel_stats(k) for k in KERNELS}


# DRAM bytes of the cluster tridiagonalisation per algorithmic byte (each
# block read once, 8 n^2), from the ncu capture of the small profiling case:
# 6.010 MB read, 0 written (the results stay in L2), against 5.913 MB.
TRDC_TRAFFIC_RATIO = 6.010368 / 5.912680


def roofline(ctx, ks, torch, dev):
    """Roofline of the kernel with the most device time in `ks`: achieved =
    algorithmic work of its launches (stated by the launching host code) /
    their CUDA-event time."""
    peaks = load_peaks()
    name, (nl, ms) = max(ks.items(), key=lambda kv: kv[1][1])
    if not nl or ms <= 0:
        return None
    work = ctx.kernel_work(name)
    if name == "trd_panel":
        # symv bytes (each column's trailing block read once) per second,
        # against the HBM copy rate for scale only: the trailing block is
        # re-read from L2 (85 % hit rate, 0.6 % of DRAM peak in the ncu
        # capture) and the kernel waits at grid barriers, so it is bound by
        # barrier latency, not by HBM
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = work / (ms / 1000.0) / 1e9
        return {"kernel": name, "bound": "latency (grid barriers; trailing block L2-resident)",
                "achieved": achieved, "peak": peak,
                "peak_source": ("measured" if "hbm_gbs" in peaks else "fallback")
                + " HBM copy rate, for scale (not the binding limit)",
                "unit": "GB/s", "frac": achieved / peak, "traffic": None, "launches": nl,
                "avg_launch_ms": ms / nl, "algorithmic_bytes_per_launch": work / nl}
    if name == "trd_cluster":
        # (4/3) n^3 flops per block on the FP64 pipe (B200's FP64 vector and
        # tensor rates are the same; the measured DGEMM rate is the peak)
        peak = fp64_gemm_peak(torch, dev)
        achieved = work / (ms / 1000.0) / 1e12
        hbm = ctx.kernel_work("trd_cluster_hbm")
        return {"kernel": name, "bound": "fp64", "achieved": achieved, "peak": peak,
                "peak_source": "measured cuBLAS DGEMM 8192^3 in this run", "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": TRDC_TRAFFIC_RATIO * hbm / nl,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the small-case capture "
                                  "(3 blocks, n = 402..580) = %.3f x 8 n^2 per block, scaled to this run's "
                                  "blocks" % TRDC_TRAFFIC_RATIO,
                "algorithmic_bytes_per_launch": hbm / nl, "launches": nl, "avg_launch_ms": ms / nl,
                "algorithmic_flops_per_launch": work / nl}
    if name.startswith("gemm_f64"):
        peak = fp64_gemm_peak(torch, dev)
        achieved = work / (ms / 1000.0) / 1e12
        return {"kernel": name, "bound": "tensor", "achieved": achieved, "peak": peak,
                "peak_source": "measured cuBLAS DGEMM 8192^3 in this run (FP64 tensor pipe)", "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None, "launches": nl, "avg_launch_ms": ms / nl,
                "algorithmic_flops_per_launch": work / nl}
    return {"kernel": name, "launches": nl, "avg_launch_ms": ms / nl, "bound": None}


# ---------------------------------------------------------------------------
# served stream
# ---------------------------------------------------------------------------
def stream_waves(waves):
    """The first `waves` x 32 requests of the served stream (256 requests);
    further waves repeat it with fresh eps_d / Nkeep draws."""
    import serve
    out = []
    rep = 0
    while len(out) < waves * WAVE:
        out += serve.stream(seed=serve.SEED + 1000 * rep)
        rep += 1
    return out[:waves * WAVE]


def keep_mix(reqs):
    n = len(reqs)
    return {k: sum(1 for r in reqs if r.keep == k) / n for k in sorted({r.keep for r in reqs})}


def one_per_keep(reqs):
    seen, out = set(), []
    for r in reqs:
        if r.keep not in seen:
            seen.add(r.keep)
            out.append(r)
    return sorted(out, key=lambda r: r.keep)


def spectra_rel_err(ref_reqs, reqs):
    """Largest relative difference per bin (bins above 1e-6 of each
    spectrum's largest) between the .bin spectra of two passes of the same
    requests."""
    worst = 0.0
    for a, b in zip(ref_reqs, reqs):
        for name in os.listdir(a.outdir):
            if not name.endswith(".bin"):
                continue
            x = np.fromfile(os.path.join(a.outdir, name), dtype="<f8").reshape(-1, 2)
            y = np.fromfile(os.path.join(b.outdir, name), dtype="<f8").reshape(-1, 2)
            dx, dy = dict(zip(x[:, 0], x[:, 1])), dict(zip(y[:, 0], y[:, 1]))
            wmax = max(abs(v) for v in dx.values()) if dx else 0.0
            for k, v in dx.items():
                if abs(v) >= 1e-6 * wmax and v != 0.0:
                    worst = max(worst, abs(dy.get(k, 0.0) - v) / abs(v))
    return worst


def bench_config(reqs):
    """The workload description both arms print (identical, so that the two
    lines describe the same configuration)."""
    mix = keep_mix(reqs)
    return {"workload": "served SIAM-QS z-averaging stream, FDM A(omega)",
            "model": "SIAM, QS symmetry, flat band, U=0.2, Gamma=0.02, Lambda=2, Nmax=40",
            "stream": "z=k/8 (k=1..8) x 32 seeded eps_d in [-0.2,0]; Nkeep seeded from {200,500,1000,2000}",
            "spectrum": "FDM A_d-A_d at T=1e-6, 50 bins per decade",
            "runs": len(reqs), "step": "one wave of %d requests of the stream, in stream order" % WAVE,
            "nkeep_mix": " ".join("%d:%.3f" % (k, f) for k, f in sorted(mix.items())),
            "arrivals": "all queued at t=0 (value, e2e); Poisson at %.0f%% of capacity for the latency"
                        % (100 * LOAD),
            "l2": "inputs larger than L2: each run's eigenvector and operator blocks stay in HBM across its "
                  "40 steps, and the runs in flight hold GBs"}


def mix_rate(per_keep_s, mix):
    """Runs/hour of a stream with Nkeep fractions `mix`, one run at a time."""
    return 3600.0 / sum(f * per_keep_s[k] for k, f in mix.items())


def max_over_ranks(dist, values, device):
    """Max over the ranks of each value (the timed spans of the replicas)."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_value(world, runs, span_s):
    """Whole-job runs/hour of `world` replicas that each served `runs` runs,
    timed as the slowest replica's span."""
    return world * 3600.0 * runs / span_s


def run_ours(args, rank, world):
    import torch

    import nrgb
    import serve
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    tmp = tempfile.mkdtemp(prefix="nrgb_bench_")
    try:
        reqs = serve.prepare(stream_waves(args.steps), os.path.join(tmp, "timed"))
        mix = keep_mix(reqs)
        warm = serve.prepare(copy.deepcopy([r for r in reqs if r.keep == min(mix)][:args.warmup] or reqs[:args.warmup]),
                             os.path.join(tmp, "warm"))
        lat = serve.prepare(copy.deepcopy(reqs[:min(LAT_RUNS, len(reqs))]), os.path.join(tmp, "lat"))
        lat_low = serve.prepare(copy.deepcopy(reqs[:min(LAT_RUNS, len(reqs))]), os.path.join(tmp, "lat_low"))
        prof = serve.prepare(copy.deepcopy(reqs[:min(WAVE, len(reqs))]), os.path.join(tmp, "prof"))
        ctx = nrgb.Context(local)  # launch accounting and the plain path
        srv = nrgb.Server(local, max_runs=args.max_runs, batch_window_us=2000.0)
        serve.serve(srv, warm, 0.0)
        # ---- profiled pass (untimed): one wave with every launch timed, for
        # the kernel shares and the dominant kernel.  Timing every launch
        # records two CUDA events per launch from all worker threads and
        # slowed the served stream by about a quarter, so the timed pass
        # below times only the dominant kernel. ----
        ctx.profile(True)
        serve.serve(srv, prof, 0.0)
        ks_all = kernel_table(ctx)
        ctx.profile(False)
        top = max(ks_all.items(), key=lambda kv: kv[1][1])[0]
        if dist:
            dist.barrier()
        # ---- timed: the stream, all requests queued at t = 0 ----
        clocks = ClockSampler(local)
        clocks.start()
        ctx.profile(True, only=top + ("*" if top == "assemble" else ""))
        res = serve.serve(srv, reqs, 0.0)
        launches, _ = ctx.kernel_stats("*")
        ks = kernel_table(ctx)
        work = {k: ctx.kernel_work(k) for k in ("trd_panel", "gemm_f64*")}
        clk = clocks.stop()
        roof = roofline(ctx, ks, torch, dev)
        ctx.profile(False)
        span, cspan = res["span_s"], res["client_span_s"]
        if dist:
            span, cspan = max_over_ranks(dist, [span, cspan], dev)
        value = replica_value(world, len(reqs), span)
        e2e_value = replica_value(world, len(reqs), cspan)
        # ---- latency under Poisson arrivals near capacity ----
        latres = serve.serve(srv, lat, LOAD * len(reqs) / res["span_s"])
        # the same at half the capacity: time-to-spectrum without a queue
        # (near capacity a busy host can leave the server short of the
        # arrival rate, and p99 then measures the growing queue)
        latlow = serve.serve(srv, lat_low, LOAD_LOW * len(reqs) / res["span_s"])
        # ---- the same stream in split precision (INT8-slice products, 8
        # slices), all queued at t = 0, and its spectra against the FP64 pass ----
        split = None
        if not args.no_split:
            sreqs = serve.prepare(copy.deepcopy(reqs), os.path.join(tmp, "split"))
            for r in sreqs:
                with open(os.path.join(r.workdir, "param"), "a") as fh:
                    fh.write("gemm_slices=8\n")
            sres = serve.serve(srv, sreqs, 0.0)
            sspan = sres["span_s"]
            if dist:
                sspan = max_over_ranks(dist, [sspan], dev)[0]
            split = {"value": replica_value(world, len(sreqs), sspan),
                     "max_spectra_rel_err": spectra_rel_err(reqs, sreqs)}
        cnt = srv.counters()
        srv.close()
        # ---- plain: one run at a time (batched per step, and per block) ----
        sample = serve.prepare(copy.deepcopy(one_per_keep(reqs)), os.path.join(tmp, "plain"))
        pl = serve.plain(sample, local)
        pb = serve.plain(sample, local, per_block=True)
        plain_rate = mix_rate(pl["per_keep_s"], mix)
        per_block_rate = mix_rate(pb["per_keep_s"], mix)
        # ---- microbenchmark (40-block step) ----
        micro = None if args.no_micro else run_micro(ctx, torch, dev, steps=args.micro_steps)
        ctx.close()
        runs = res["runs"]
        waves = args.steps
        h2d = sum(r["h2d_bytes"] for r in runs) / waves
        d2h = sum(r["d2h_bytes"] for r in runs) / waves
        tot_ms = sum(v[1] for v in ks_all.values())
        detail = {
            "latency_s": {"p50": latres["p50_latency_s"], "p99": latres["p99_latency_s"],
                          "rate_hz": latres["rate_hz"], "runs": latres["n"],
                          "runs_per_hour": latres["runs_per_hour"],
                          "closed_loop_p50": res["p50_latency_s"], "closed_loop_p99": res["p99_latency_s"]},
            "latency_s_half_load": {"p50": latlow["p50_latency_s"], "p99": latlow["p99_latency_s"],
                                    "rate_hz": latlow["rate_hz"], "runs": latlow["n"],
                                    "runs_per_hour": latlow["runs_per_hour"]},
            "plain": {"per_keep_s_batched_steps": pl["per_keep_s"], "per_keep_s_per_block": pb["per_keep_s"],
                      "sample": "one run per Nkeep, one after another through nrgb_run; runs/hour for the "
                                "stream's Nkeep mix"},
            "server": {k: cnt[k] for k in ("eig_calls", "eig_requests", "eig_blocks", "peak_running",
                                           "peak_admitted_bytes", "budget_bytes")},
            "kernel_time_share": {k: round(v[1] / tot_ms, 4) for k, v in ks_all.items() if tot_ms and v[1] / tot_ms > 0.001},
            "kernel_time_share_source": "profiled pass of one wave (%d requests) before the timed region, every "
                                        "launch timed; the timed pass times only %s" % (len(prof), top),
            "work": work,
        }
        line = {
            "metric": METRIC, "value": value, "unit": "runs/hour", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * span / waves, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(reqs),
            "clocks": clk,
            # end to end through the public API: the stream on the client's
            # clock (result files read back), the time-to-spectrum under
            # Poisson arrivals, and the plain FP64 path through nrgb_run
            "e2e": {"value": e2e_value, "unit": "runs/hour", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "readback_bytes": res["readback_bytes"],
                    "p50_latency_s": latres["p50_latency_s"], "p99_latency_s": latres["p99_latency_s"],
                    "latency_rate_hz": latres["rate_hz"], "latency_runs": latres["n"],
                    "plain_per_block_runs_per_hour": per_block_rate,
                    "plain_batched_runs_per_hour": plain_rate,
                    "served_over_per_block": value / world / per_block_rate,
                    "served_over_plain_batched": value / world / plain_rate,
                    **({"served_split8_runs_per_hour": split["value"],
                        "served_split8_over_per_block": split["value"] / world / per_block_rate,
                        "split8_max_spectra_rel_err": split["max_spectra_rel_err"]} if split else {}),
                    "server_slots": args.max_runs},
            "gpu_launches": int(launches),
            "roofline": roof,
        }
        if micro:
            detail["microbench"] = micro
        if rank == 0 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(reqs, os.path.join(tmp, "cpu"), args.cpu_budget)
        if rank == 0:
            # the details go to stderr (one line); stdout carries the one
            # compact result line
            print("# bench detail " + json.dumps(detail), file=sys.stderr, flush=True)
            if args.detail:
                with open(args.detail, "w") as fh:
                    json.dump({"line": line, "detail": detail}, fh, indent=1)
            print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# CPU: the reference's algorithm (the oracle) on the host cores
# ---------------------------------------------------------------------------
# The reference's CPU path is timed in the two settings of its OpenMP build
# and the faster is used: blocks diagonalised concurrently, one per core with
# one BLAS thread each (OpenMP over blocks, src/nrg.cc:2484-2507), or one
# block at a time with LAPACK/BLAS threaded over all cores.  Both use the
# reference's faster eigensolver option diag=dsyevr (src/read-input.cc:16-33,
# src/diag.h:93-160; dsyev below dsyevrlimit = 100), which makes the CPU
# baseline stronger than the default dsyev.
CPU_SETTINGS = ("omp_blocks", "blas_threads")


def _cpu_prepare(reqs, root):
    import serve
    reqs = serve.prepare(copy.deepcopy(reqs), root)
    for r in reqs:
        with open(os.path.join(r.workdir, "param"), "a") as fh:
            fh.write("diag=dsyevr\n")
    return reqs


def oracle_run(req, setting, cores):
    """Seconds of one run of the CPU oracle (the reference's algorithm) on
    `cores` host threads in `setting`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import nrg_oracle
    from threadpoolctl import threadpool_limits
    t0 = time.perf_counter()
    if setting == "omp_blocks":
        nrg_oracle.Oracle(req.workdir, threads=cores).run(req.outdir)
    else:
        with threadpool_limits(limits=cores, user_api="blas"):
            nrg_oracle.Oracle(req.workdir, threads=1).run(req.outdir)
    return time.perf_counter() - t0


def pick_setting(req, cores):
    """Time `req` in both settings; returns (faster setting, seconds of each)."""
    t = {st: oracle_run(req, st, cores) for st in CPU_SETTINGS}
    return min(t, key=t.get), t


def cpu_baseline(reqs, root, budget_s):
    """Bounded sample for the GPU line: one run per Nkeep class in the faster
    setting, ascending, while the budget lasts; a class past the budget is
    extrapolated from the previous one as Nkeep^3 (said in `sample`)."""
    cores = os.cpu_count() or 1
    sample = _cpu_prepare(one_per_keep(reqs), root)
    calib = [r for r in sample if r.keep <= 500] or sample[:1]
    setting, tset = pick_setting(calib[-1], cores)
    times, how = {}, {}
    spent = sum(tset.values())
    prev = None
    for r in sample:
        if prev is not None and (times[prev] * (r.keep / prev) ** 3 > budget_s - spent):
            times[r.keep] = times[prev] * (r.keep / prev) ** 3
            how[r.keep] = "extrapolated from Nkeep=%d as Nkeep^3" % prev
        else:
            times[r.keep] = oracle_run(r, setting, cores)
            spent += times[r.keep]
            how[r.keep] = "measured"
        prev = r.keep
    return {"value": mix_rate(times, keep_mix(reqs)), "unit": "runs/hour", "cores": cores, "kind": "port",
            "setting": setting, "diag": "dsyevr",
            "sample": "one run per Nkeep through the CPU oracle, %s on %d threads, diag=dsyevr: %s; runs/hour for "
                      "the stream's Nkeep mix (the reference arm measures every class)"
                      % (setting, cores, ", ".join("Nkeep=%d %.1f s (%s)" % (k, times[k], how[k]) for k in sorted(times))),
            **{"s_nkeep%d" % k: times[k] for k in sorted(times)}}


def run_reference(args, rank, world):
    """The reference's CPU path (the oracle) on the host cores, same stream:
    warm-up picks the faster of the two settings on a Nkeep <= 1000 run and
    runs W runs of the smallest class; each timed step is one request of the
    stream in stream order (every Nkeep class measured, none extrapolated)."""
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    reqs = stream_waves(args.steps)  # the GPU arm's stream (same config)
    timed = reqs[:args.steps]
    tmp = tempfile.mkdtemp(prefix="nrgb_ref_")
    try:
        cal = [r for r in reqs if r.keep <= 1000]
        cal = max(cal, key=lambda r: r.keep) if cal else reqs[0]
        setting, tset = pick_setting(_cpu_prepare([cal], os.path.join(tmp, "cal"))[0], cores)
        kmin = min(r.keep for r in reqs)
        small = [r for r in reqs if r.keep == kmin][:1]
        for i in range(args.warmup):
            oracle_run(_cpu_prepare(small, os.path.join(tmp, "w%d" % i))[0], setting, cores)
        work = _cpu_prepare(timed, os.path.join(tmp, "timed"))
        step_s = [oracle_run(r, setting, cores) for r in work]
        total = sum(step_s)
        value = 3600.0 * len(work) / total
        per_keep = {}
        for r, t in zip(work, step_s):
            per_keep.setdefault(r.keep, []).append(t)
        mean = {k: statistics.mean(v) for k, v in sorted(per_keep.items())}
        sample = ("the first %d requests of the stream, one after another through the CPU oracle, %s on %d "
                  "threads (faster of omp_blocks %.1f s / blas_threads %.1f s on a Nkeep=%d run), diag=dsyevr; "
                  "mean s per run: %s" % (len(work), setting, cores, tset["omp_blocks"], tset["blas_threads"],
                                         cal.keep, ", ".join("Nkeep=%d %.1f" % (k, v) for k, v in mean.items())))
        line = {"metric": METRIC, "value": value, "unit": "runs/hour", "impl": "reference", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / len(work),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": bench_config(reqs),
                "cpu_baseline": {"value": value, "unit": "runs/hour", "cores": cores, "kind": "port",
                                 "setting": setting, "diag": "dsyevr", "sample": sample,
                                 **{"s_nkeep%d" % k: v for k, v in mean.items()}},
                "e2e": {"value": value, "unit": "runs/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                        "p50_latency_s": float(np.percentile(step_s, 50)),
                        "p99_latency_s": float(np.percentile(step_s, 99))}}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


# ---------------------------------------------------------------------------
# microbenchmark: 40 dense blocks per step
# ---------------------------------------------------------------------------
def step_sizes(step):
    """Block sizes of a step: log-uniform on [16, 4096] (NMAX caps them for
    small profiling cases)."""
    rng = np.random.default_rng(SEED + step)
    return [min(NMAX, int(round(math.exp(x)))) for x in rng.uniform(math.log(16), math.log(4096), NBLOCKS)]


def pairs(nb=NBLOCKS):
    bra, ket = [], []
    for k in range(nb):
        for _ in range(NOPS_PER_PAIR):
            bra.append(k)
            ket.append((k + 1) % nb)
    return bra, ket


def device_batch(torch, step, dev):
    ns = step_sizes(step)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 1000 + step)
    H = []
    for n in ns:
        G = torch.randn(n, n, generator=g, device=dev, dtype=torch.float64)
        Q, R = torch.linalg.qr(G)
        Q = Q * torch.sign(torch.diagonal(R))
        sgn = torch.randint(0, 2, (n,), generator=g, device=dev).to(torch.float64) * 2 - 1
        lam = torch.logspace(-12, 1, n, device=dev, dtype=torch.float64) * sgn
        A = (Q * lam) @ Q.T
        H.append(((A + A.T) / 2).contiguous())
    bra, ket = pairs()
    O = [torch.randn(ns[k], ns[b], generator=g, device=dev, dtype=torch.float64).contiguous()
         for b, k in zip(bra, ket)]  # torch (nk x nb) row-major == column-major nb x nk
    return ns, H, O


def run_micro(ctx, torch, dev, steps):
    """Batched eigensolve + recalc of 40 blocks per step, against one solver
    call per block; device-resident inputs; CUDA events on the launch stream."""
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    bra, ket = pairs()
    batches = [device_batch(torch, s, dev) for s in range(steps + 1)]
    nmax_tot = max(sum(n * n for n in b[0]) for b in batches)
    A = torch.empty(nmax_tot, device=dev, dtype=torch.float64)
    Zb = torch.empty(nmax_tot, device=dev, dtype=torch.float64)
    Wb = torch.empty(NBLOCKS * 4096, device=dev, dtype=torch.float64)
    omax = max(sum(b[0][bb] * b[0][kk] for bb, kk in zip(bra, ket)) for b in batches)
    Ob = torch.empty(omax, device=dev, dtype=torch.float64)

    def step(i):
        ns, H, O = batches[i]
        a, z, w, o = [], [], [], []
        pa = pw = po = 0
        for h, n in zip(H, ns):
            A[pa:pa + n * n].copy_(h.view(-1))
            a.append(A.data_ptr() + 8 * pa)
            z.append(Zb.data_ptr() + 8 * pa)
            w.append(Wb.data_ptr() + 8 * pw)
            pa += n * n
            pw += n
        for b, k in zip(bra, ket):
            o.append(Ob.data_ptr() + 8 * po)
            po += ns[b] * ns[k]
        ctx.eig_recalc_step_dev(ns, a, w, z, bra, ket, [x.data_ptr() for x in O], o, stream=sh)

    out = {"workload": "40 blocks per step, n log-uniform in [16, 4096], lambda logspace(-12, 1) with random "
                       "signs, 6 operator blocks per block pair; eigensolve + 240 basis changes",
           "steps": steps}
    for mode, key in ((0, "batched"), (1, "per_block")):
        ctx.set_eig_mode(mode)
        step(0)
        torch.cuda.synchronize()
        if mode == 0:
            ctx.profile(True)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for i in range(steps):
            step(1 + i)
        t1.record(stream)
        torch.cuda.synchronize()
        out[key + "_ms_per_step"] = t0.elapsed_time(t1) / steps
        if mode == 0:
            out["check"] = check_micro(torch, batches[steps], A, Zb, Wb, Ob, bra, ket)
            ks = kernel_table(ctx)
            out["roofline"] = roofline(ctx, {k: v for k, v in ks.items() if k == "trd_panel"}, torch, dev)
            tot = sum(v[1] for v in ks.values())
            out["kernel_time_share"] = {k: round(v[1] / tot, 4) for k, v in ks.items() if tot and v[1] / tot > 0.001}
            out["gemm_ms_per_step_by_site"] = {k: round(v[1] / steps, 3) for k, v in ks.items() if k.startswith("gemm")}
            ctx.profile(False)
    ctx.set_eig_mode(0)
    out["batched_over_per_block"] = out["per_block_ms_per_step"] / out["batched_ms_per_step"]
    return out


def check_micro(torch, batch, A, Zb, Wb, Ob, bra, ket):
    """Checks of the last timed step's results: per block, the eigenvalue sum
    against the trace and the ordering; the residual |H z - w z| and the
    orthonormality of the eigenvectors of the largest block; every basis
    change of the largest block against torch FP64 (Z_b^T O Z_k)."""
    ns, H, O = batch
    offs, woffs, ooffs = [], [], []
    pa = pw = po = 0
    for n in ns:
        offs.append(pa)
        woffs.append(pw)
        pa += n * n
        pw += n
    for b, k in zip(bra, ket):
        ooffs.append(po)
        po += ns[b] * ns[k]
    worst_tr = 0.0
    for n, h, pw_ in zip(ns, H, woffs):
        w = Wb[pw_:pw_ + n]
        assert bool(torch.all(w[1:] >= w[:-1])), "eigenvalues not ascending"
        tr = torch.trace(h).item()
        worst_tr = max(worst_tr, abs(w.sum().item() - tr) / (1.0 + h.abs().sum().item() / n))
    big = max(range(len(ns)), key=lambda i: ns[i])
    n = ns[big]
    Z = Zb[offs[big]:offs[big] + n * n].view(n, n).t()  # column r = eigenvector r
    w = Wb[woffs[big]:woffs[big] + n]
    nrm = w.abs().max().item()
    res = ((H[big] @ Z - Z * w).abs().max().item()) / (nrm * n)
    orth = (Z.T @ Z - torch.eye(n, dtype=torch.float64, device=Z.device)).abs().max().item() / n
    rec = 0.0
    for o, (b, k) in enumerate(zip(bra, ket)):
        if b != big and k != big:
            continue
        nb, nk = ns[b], ns[k]
        Zb_ = Zb[offs[b]:offs[b] + nb * nb].view(nb, nb).t()
        Zk_ = Zb[offs[k]:offs[k] + nk * nk].view(nk, nk).t()
        op = O[o].t()  # nb x nk
        ref = Zb_.T @ op @ Zk_
        got = Ob[ooffs[o]:ooffs[o] + nb * nk].view(nk, nb).t()
        rec = max(rec, (got - ref).abs().max().item() / (ref.abs().max().item() + 1.0))
    ok = worst_tr <= 1e-12 and res <= 1e-13 and orth <= 1e-13 and rec <= 1e-12
    if not ok:
        raise RuntimeError("microbenchmark results failed their checks: trace %.3g residual %.3g orth %.3g "
                           "recalc %.3g" % (worst_tr, res, orth, rec))
    return {"trace_rel": worst_tr, "largest_block": n, "residual_per_n": res, "orth_per_n": orth,
            "recalc_rel": rec}


def run_micro_only(args):
    """Only the microbenchmark (profiling runs)."""
    import torch

    import nrgb
    dev = torch.device("cuda", 0)
    ctx = nrgb.Context(0)
    print(json.dumps(run_micro(ctx, torch, dev, steps=args.steps)), flush=True)
    ctx.close()
    return 0


def run_split_micro(edge, slices, nprob):
    """Split-precision grouped GEMM (INT8 slices on tcgen05) against the FP64
    DMMA grouped GEMM on `nprob` problems of edge^3, device-resident inputs;
    CUDA events on the launch stream; the split result is checked against
    the FP64 one."""
    import torch

    import nrgb
    dev = torch.device("cuda", 0)
    ctx = nrgb.Context(0)
    g = torch.Generator(device=dev).manual_seed(SEED)
    A = [torch.randn(edge, edge, generator=g, device=dev, dtype=torch.float64) for _ in range(nprob)]
    B = [torch.randn(edge, edge, generator=g, device=dev, dtype=torch.float64) for _ in range(nprob)]
    C1 = [torch.empty(edge, edge, device=dev, dtype=torch.float64) for _ in range(nprob)]
    C2 = [torch.empty(edge, edge, device=dev, dtype=torch.float64) for _ in range(nprob)]
    terms = [nrgb.GemmTerm(a.data_ptr(), b.data_ptr(), edge, edge, edge, 0, 0, 1.0) for a, b in zip(A, B)]
    o1 = [nrgb.GemmOut(c.data_ptr(), edge, edge, edge, 0.0, i, 1) for i, c in enumerate(C1)]
    o2 = [nrgb.GemmOut(c.data_ptr(), edge, edge, edge, 0.0, i, 1) for i, c in enumerate(C2)]
    st = torch.cuda.current_stream(dev)
    out = {"edge": edge, "problems": nprob, "slices": slices}
    fl = 2.0 * edge ** 3 * nprob
    for key, fn in (("fp64", lambda: ctx.gemm_grouped_dev(o1, terms, stream=st.cuda_stream)),
                    ("split", lambda: ctx.gemm_grouped_split_dev(slices, o2, terms, stream=st.cuda_stream))):
        fn()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(st)
            fn()
            t1.record(st)
            torch.cuda.synchronize()
            best = min(best, t0.elapsed_time(t1))
        out[key + "_ms"] = best
        out[key + "_tflops"] = fl / best / 1e9
    # the split call includes slicing the operands; its INT8 work is
    # S(S+1)/2 products of the same shape
    out["int8_tops"] = fl * slices * (slices + 1) / 2 / out["split_ms"] / 1e9
    err = max(((x - y).abs().max() / (y.abs().max() + 1.0)).item() for x, y in zip(C2, C1))
    out["max_rel_diff_vs_fp64"] = err
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


def run_gemm_micro():
    """Grouped FP64 GEMM (the kernel NRGB_GEMM_PIPE selects in this process)
    on square problems in all four transpose combinations, and cuBLAS DGEMM
    (torch.bmm) on the same untransposed problems; device-resident inputs,
    CUDA events on the launch stream, best of 5.  Prints one JSON object of
    TF/s per case."""
    import torch

    import nrgb
    dev = torch.device("cuda", 0)
    ctx = nrgb.Context(0)
    st = torch.cuda.current_stream(dev)
    g = torch.Generator(device=dev).manual_seed(SEED)

    def best_ms(fn):
        fn()
        torch.cuda.synchronize()
        best = 1e30
        for _ in range(5):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(st)
            fn()
            t1.record(st)
            torch.cuda.synchronize()
            best = min(best, t0.elapsed_time(t1))
        return best

    forms = {"0": "register-staged", "3": "pipelined, K step 16, 3 stages", "4": "pipelined, K step 16, 4 stages",
             "232": "pipelined, K step 32, 2 stages", "332": "pipelined, K step 32, 3 stages"}
    out = {"kernel": forms.get(os.environ.get("NRGB_GEMM_PIPE") or "3", "pipelined, K step 16, 3 stages")}
    for edge, nprob, nseg in ((2048, 4, 1), (1024, 16, 1), (512, 64, 1), (384, 64, 3), (256, 128, 2)):
        for ta, tb in ((0, 0), (1, 0), (0, 1), (1, 1)):
            A = [torch.randn(edge, edge, generator=g, device=dev, dtype=torch.float64) for _ in range(nprob * nseg)]
            B = [torch.randn(edge, edge, generator=g, device=dev, dtype=torch.float64) for _ in range(nprob * nseg)]
            C = [torch.empty(edge, edge, device=dev, dtype=torch.float64) for _ in range(nprob)]
            terms = [nrgb.GemmTerm(a.data_ptr(), b.data_ptr(), edge, edge, edge, ta, tb, 1.0) for a, b in zip(A, B)]
            outs = [nrgb.GemmOut(c.data_ptr(), edge, edge, edge, 0.0, i * nseg, nseg) for i, c in enumerate(C)]
            ms = best_ms(lambda: ctx.gemm_grouped_dev(outs, terms, stream=st.cuda_stream))
            key = "%dx%d^3 (%d segments) t%d%d" % (nprob, edge, nseg, ta, tb)
            out[key] = round(2.0 * edge ** 3 * nprob * nseg / ms / 1e9, 2)
            if ta == 0 and tb == 0:
                Ab, Bb = torch.stack(A[:nprob]), torch.stack(B[:nprob])
                ms2 = best_ms(lambda: torch.bmm(Ab, Bb))
                out["cublas %dx%d^3" % (nprob, edge)] = round(2.0 * edge ** 3 * nprob / ms2 / 1e9, 2)
                del Ab, Bb
            del A, B, C
            torch.cuda.empty_cache()
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


def run_configs(args):
    """Wall time of one run of each workload through nrgb_run on the GPU
    (batched eigensolves per step; one eigensolver call per block; split
    precision where it applies) and of the CPU oracle on the host cores
    (faster of the two settings, diag=dsyevr) where that fits in minutes.
    Prints one JSON object."""
    import nrgb
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import nrg_cases as cases
    cores = os.cpu_count() or 1
    out = {"cores": cores}
    tmp = tempfile.mkdtemp(prefix="nrgb_cfg_")
    try:
        for name, cpu in (("siam_nmax30", True), ("siam_c4", True), ("kondo2ch_full", False)):
            wd = cases.make_case(name, os.path.join(tmp, name))
            rec = {}
            for mode, key in ((0, "gpu_batched_s"), (1, "gpu_per_block_s")):
                ctx = nrgb.Context(0)
                ctx.set_eig_mode(mode)
                od = os.path.join(tmp, name + "_out%d" % mode)
                os.makedirs(od, exist_ok=True)
                t0 = time.perf_counter()
                ctx.run(wd, od)
                rec[key] = time.perf_counter() - t0
                ctx.close()
            if name == "siam_c4":
                import shutil as _sh
                wd2 = os.path.join(tmp, name + "_split")
                _sh.copytree(wd, wd2)
                with open(os.path.join(wd2, "param"), "a") as fh:
                    fh.write("gemm_slices=8\n")
                ctx = nrgb.Context(0)
                od = os.path.join(tmp, name + "_outsplit")
                os.makedirs(od, exist_ok=True)
                t0 = time.perf_counter()
                ctx.run(wd2, od)
                rec["gpu_batched_split8_s"] = time.perf_counter() - t0
                ctx.close()
            if cpu and not args.no_cpu_baseline:
                import serve
                req = serve.Request(z=1.0, eps_d=0.0, keep=0, workdir=wd, outdir=os.path.join(tmp, name + "_cpu"))
                with open(os.path.join(wd, "param"), "a") as fh:
                    fh.write("diag=dsyevr\n")
                rec["cpu_oracle_s"] = oracle_run(req, "omp_blocks", cores)
            out[name] = rec
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    print(json.dumps(out), flush=True)
    return 0


def run_one_case(name):
    """One NRG run of a test workload (tests/nrg_cases.py) through nrgb_run,
    for profiling the whole step (assembly, eigensolver, truncation,
    recalculation, density matrices, spectra)."""
    import nrgb
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import nrg_cases as cases
    tmp = tempfile.mkdtemp(prefix="nrgb_one_")
    try:
        wd = cases.make_case(name, os.path.join(tmp, "in"))
        od = os.path.join(tmp, "out")
        os.makedirs(od)
        ctx = nrgb.Context(0)
        st = ctx.run(wd, od)
        ctx.close()
        print(json.dumps({"case": name, "wall_s": st["wall_s"], "launches": st["launches"]}), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


def run_ncu_small(nmax):
    """Small profiling case (no torch on the GPU): 12 blocks with sizes up to
    `nmax` and their 72 operators through the host-buffer C ABI, twice."""
    import nrgb
    rng = np.random.default_rng(SEED)
    ns = [int(x) for x in np.linspace(48, nmax, 12)]
    bra, ket = pairs(len(ns))
    H = []
    for n in ns:
        X = rng.standard_normal((n, n))
        H.append(np.asfortranarray((X + X.T) / 2))
    O = [np.asfortranarray(rng.standard_normal((ns[b], ns[k]))) for b, k in zip(bra, ket)]
    W = [np.empty(n) for n in ns]
    R = [np.empty((ns[b], ns[k]), order="F") for b, k in zip(bra, ket)]
    ctx = nrgb.Context(0)
    for _ in range(2):
        ctx.eig_recalc_step(ns, [h.ctypes.data for h in H], [w.ctypes.data for w in W], None, bra, ket,
                            [o.ctypes.data for o in O], [r.ctypes.data for r in R])
    for h, w in zip(H, W):
        assert abs(np.sum(w) - np.trace(h)) <= 1e-9 * (1 + np.abs(h).sum())
    ctx.close()
    print(json.dumps({"ncu_small": nmax, "blocks": ns}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4, help="waves of 32 requests (served); steps (--micro)")
    ap.add_argument("--warmup", type=int, default=3, help="untimed warm-up runs (at least 3)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--max-runs", type=int, default=MAX_RUNS, help="worker slots of the run server")
    ap.add_argument("--cpu-budget", type=float, default=40.0, help="seconds of oracle work for cpu_baseline")
    ap.add_argument("--ref-budget", type=float, default=40.0, help="seconds of oracle work per reference step")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-micro", action="store_true", help="skip the 40-block microbenchmark")
    ap.add_argument("--no-split", action="store_true", help="skip the split-precision pass of the stream")
    ap.add_argument("--micro-steps", type=int, default=20, help="steps of the 40-block microbenchmark")
    ap.add_argument("--detail", default="", help="also write the line and its details to this JSON file")
    ap.add_argument("--micro", action="store_true", help="run only the 40-block microbenchmark")
    ap.add_argument("--nmax", type=int, default=4096, help="cap on block sizes of the microbenchmark")
    ap.add_argument("--split-micro", type=int, default=0,
                    help="time the split-precision grouped GEMM against FP64 on problems of this edge")
    ap.add_argument("--gemm-micro", action="store_true",
                    help="time the grouped FP64 GEMM in all transpose combinations against cuBLAS")
    ap.add_argument("--slices", type=int, default=8)
    ap.add_argument("--one-run", default="", help="one nrgb_run of a test workload (profiling)")
    ap.add_argument("--configs", action="store_true",
                    help="time one run of each workload on the GPU and (where it fits) on the CPU oracle")
    ap.add_argument("--nprob", type=int, default=4)
    ap.add_argument("--ncu-small", type=int, default=0,
                    help="run only the small profiling case with blocks up to this size (no torch GPU work)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global NMAX
    NMAX = args.nmax
    if args.ncu_small:
        return run_ncu_small(args.ncu_small)
    if args.split_micro:
        return run_split_micro(args.split_micro, args.slices, args.nprob)
    if args.gemm_micro:
        return run_gemm_micro()
    if args.configs:
        return run_configs(args)
    if args.one_run:
        return run_one_case(args.one_run)
    if args.micro:
        return run_micro_only(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world)


if __name__ == "__main__":
    sys.exit(main())
