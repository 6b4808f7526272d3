#!/usr/bin/env python3
"""Benchmark of the NRG step hot path on B200 (one JSON line on stdout).

Workload: the batched eigensolve + operator-recalculation step of an NRG
iteration at benchmark scale: each step has 40 dense symmetric blocks with
sizes drawn log-uniformly from [16, 4096] (seeded), each block
H = Q diag(lambda) Q^T with lambda log-spaced from 1e-12 to 10 with random
signs and Q orthogonal (QR of a Gaussian matrix); each block pair (k, k+1 mod
40) carries 6 standard-normal operator blocks.  One step = eigen-decomposition
of the 40 blocks + the 240 basis changes Q_k^T O Q_{k+1}.  One "run" = 20
steps; the metric is runs/hour.

  value : device-resident inputs, one batched call per step (libnrgb)
  e2e   : the same through the host-buffer C ABI (nrgb_eig_recalc_step), with
          host->device copies of the blocks/operators and device->host copies
          of the eigenvalues and recalculated operators inside the timed region
  --impl reference : the CPU path (LAPACK dsyev per block, OpenMP-style over
          blocks as the reference's diagth loop, BLAS gemm for the recalc) on
          all host cores, on a bounded sample of every step.

Multi-GPU (torchrun): the step does not shard; every rank runs an independent
replica (weak scaling) and value is the sum over ranks, timed as the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nrgljubljana-old_b200"))

METRIC = "NRG runs/hour and p50/p99 latency, served vs plain FP64 (spectra <=1e-8 rel err)"
STEPS_PER_RUN = 20
NBLOCKS = 40
NOPS_PER_PAIR = 6
SEED = 20261204  # 20261203 + config index 1


NMAX = 4096


def step_sizes(step):
    """Block sizes of a step: log-uniform on [16, 4096] (NMAX caps them for
    small profiling cases)."""
    rng = np.random.default_rng(SEED + step)
    return [min(NMAX, int(round(math.exp(x)))) for x in rng.uniform(math.log(16), math.log(4096), NBLOCKS)]


def pairs():
    bra, ket = [], []
    for k in range(NBLOCKS):
        for _ in range(NOPS_PER_PAIR):
            bra.append(k)
            ket.append((k + 1) % NBLOCKS)
    return bra, ket


def algorithmic_flops(ns):
    """eig: (14/3) n^3 per block; recalc Q_b^T O Q_k: 2 nb nk^2 + 2 nb^2 nk per operator."""
    bra, ket = pairs()
    f = sum(14.0 / 3.0 * n ** 3 for n in ns)
    f += sum(2.0 * ns[b] * ns[k] * ns[k] + 2.0 * ns[b] * ns[b] * ns[k] for b, k in zip(bra, ket))
    return f


def trd_panel_step_bytes(ns):
    """Algorithmic HBM bytes of the tridiagonalisation panel kernels of one
    step: the symmetric matrix-vector product of column c reads the trailing
    (n-c-1)^2 block once (8 bytes per element), for every block with n > 32."""
    tot = 0.0
    for n in ns:
        if n > 32:
            m = np.arange(1, n, dtype=np.float64)
            tot += 8.0 * float(np.sum(m * m))
    return tot


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

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
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        for r in self.rows:
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU path (the reference's algorithm on the host cores)
# ---------------------------------------------------------------------------
def host_block(step, k, n):
    """Synthetic block k of a step (CPU, numpy)."""
    rng = np.random.default_rng(SEED + 100000 + 1000 * step + k)
    Q, R = np.linalg.qr(rng.standard_normal((n, n)))
    Q = Q * np.sign(np.diag(R))
    lam = np.logspace(-12, 1, n) * rng.choice([-1.0, 1.0], n)
    A = (Q * lam) @ Q.T
    return np.asfortranarray((A + A.T) / 2)


def host_op(step, o, nb, nk):
    rng = np.random.default_rng(SEED + 500000 + 1000 * step + o)
    return np.asfortranarray(rng.standard_normal((nb, nk)))


CPU_SAMPLE_NMAX = 1536


def cpu_step(step, threads, budget_s):
    """The reference's CPU algorithm on one step: dsyev per block (a pool of
    `threads` workers with one BLAS thread each, as the OpenMP loop over blocks
    of src/nrg.cc:2484-2507), then the recalc GEMMs.  Blocks with
    n <= CPU_SAMPLE_NMAX are taken in a random order until `budget_s` of work
    is spent (input generation is not timed); the time is extrapolated to the
    whole step by algorithmic flops.  Returns (seconds of work, fraction of the
    step's flops done)."""
    import scipy.linalg as sla
    from concurrent.futures import ThreadPoolExecutor
    from threadpoolctl import threadpool_limits
    ns = step_sizes(step)
    order = [b for b in np.random.default_rng(SEED + 7 + step).permutation(len(ns)) if ns[b] <= CPU_SAMPLE_NMAX]
    total = algorithmic_flops(ns)
    bra, ket = pairs()
    done = 0.0
    work = 0.0
    Z = {}
    with threadpool_limits(limits=1, user_api="blas"):
        with ThreadPoolExecutor(threads) as ex:
            for c0 in range(0, len(order), threads):
                chunk = order[c0:c0 + threads]
                mats = {b: host_block(step, b, ns[b]) for b in chunk}
                t0 = time.perf_counter()
                res = list(ex.map(lambda b: sla.eigh(mats[b], driver="ev", check_finite=False), chunk))
                work += time.perf_counter() - t0
                for b, (w, v) in zip(chunk, res):
                    Z[b] = v
                    done += 14.0 / 3.0 * ns[b] ** 3
                if work > budget_s:
                    break
            jobs = [o for o, (b, k) in enumerate(zip(bra, ket)) if b in Z and k in Z]
            ops = {o: host_op(step, o, ns[bra[o]], ns[ket[o]]) for o in jobs}
            t0 = time.perf_counter()
            list(ex.map(lambda o: Z[bra[o]].T @ (ops[o] @ Z[ket[o]]), jobs))
            work += time.perf_counter() - t0
            for o in jobs:
                b, k = bra[o], ket[o]
                done += 2.0 * ns[b] * ns[k] * ns[k] + 2.0 * ns[b] * ns[b] * ns[k]
    return work, done / total


def run_reference(args, rank, world):
    threads = os.cpu_count() or 1
    if rank != 0:
        return 0
    per_step = []
    for s in range(args.warmup + args.steps):
        t, frac = cpu_step(s % STEPS_PER_RUN, threads, budget_s=args.ref_budget)
        if s >= args.warmup:
            per_step.append(t / frac)
    ms = 1000.0 * statistics.mean(per_step)
    value = 3600.0 / (STEPS_PER_RUN * ms / 1000.0)
    sample = ("blocks with n <= %d of each step in random order until %.0f s of work, extrapolated to the "
              "whole step by algorithmic flops" % (CPU_SAMPLE_NMAX, args.ref_budget))
    line = {"metric": METRIC, "value": value, "unit": "runs/hour", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "40-block eigensolve + recalc step (16..4096, log-uniform), 20 steps per run",
                       "blocks_per_step": NBLOCKS, "ops_per_pair": NOPS_PER_PAIR, "steps_per_run": STEPS_PER_RUN},
            "cpu_baseline": {"value": value, "unit": "runs/hour", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "runs/hour", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "latency_ms": {"p50": float(np.percentile(per_step, 50)) * 1000 * STEPS_PER_RUN,
                           "p99": float(np.percentile(per_step, 99)) * 1000 * STEPS_PER_RUN}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU path
# ---------------------------------------------------------------------------
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


def run_ours(args, rank, world):
    import torch
    import nrgb
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = nrgb.Context(local)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    bra, ket = pairs()
    nbatch = min(STEPS_PER_RUN, args.warmup + args.steps)
    batches = [device_batch(torch, s, dev) for s in range(nbatch)]
    # working buffers (the eigensolver destroys its input: A is refilled every step)
    nmax_tot = max(sum(n * n for n in b[0]) for b in batches)
    A = torch.empty(nmax_tot, device=dev, dtype=torch.float64)
    Zb = torch.empty(nmax_tot, device=dev, dtype=torch.float64)
    Wb = torch.empty(NBLOCKS * 4096, device=dev, dtype=torch.float64)
    omax = max(sum(b[0][bb] * b[0][kk] for bb, kk in zip(bra, ket)) for b in batches)
    Ob = torch.empty(omax, device=dev, dtype=torch.float64)

    def views(ns):
        a, z, w, o = [], [], [], []
        pa = pw = po = 0
        for n in ns:
            a.append(A.data_ptr() + 8 * pa)
            z.append(Zb.data_ptr() + 8 * pa)
            w.append(Wb.data_ptr() + 8 * pw)
            pa += n * n
            pw += n
        for b, k in zip(bra, ket):
            o.append(Ob.data_ptr() + 8 * po)
            po += ns[b] * ns[k]
        return a, z, w, o

    def step(i):
        ns, H, O = batches[i % nbatch]
        off = 0
        for h, n in zip(H, ns):
            A[off:off + n * n].copy_(h.view(-1))
            off += n * n
        a, z, w, o = views(ns)
        ctx.eig_recalc_step_dev(ns, a, w, z, bra, ket, [x.data_ptr() for x in O], o, stream=sh)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # ---- timed region (device resident) ----
    clocks = ClockSampler(local)
    clocks.start()
    ctx.profile(True)
    torch.cuda.synchronize()
    evs = []
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(args.warmup + i)
        e1.record(stream)
        evs.append((e0, e1))
    t_end.record(stream)
    torch.cuda.synchronize()
    elapsed = t_start.elapsed_time(t_end) / 1000.0
    step_ms = [a.elapsed_time(b) for a, b in evs]
    launches, _ = ctx.kernel_stats("*")
    kstats = {}
    for name in ("trd_panel", "gemm_f64*", "dc_prep", "dc_permute", "dc_secular", "dc_lowner", "dc_vectors",
                 "dc_rank", "dc_copy", "dc_leaf", "bt_T", "bt_buildV", "syev_small"):
        kstats[name.rstrip("*")] = ctx.kernel_stats(name)
    gemm_sites = {k: ctx.kernel_stats(k) for k in ("gemm_f64_trailing", "gemm_f64_dc", "gemm_f64_bt",
                                                   "gemm_f64_recalc")}
    ctx.profile(False)
    clk = clocks.stop()
    if dist:
        t = torch.tensor([elapsed], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed = float(t.item())
    ms_per_step = 1000.0 * elapsed / args.steps
    value = world * 3600.0 / (STEPS_PER_RUN * elapsed / args.steps)
    # ---- e2e through the host-buffer C ABI ----
    hb = []
    if args.no_e2e:
        nbatch_e2e = 0
    else:
        nbatch_e2e = min(nbatch, 2)
    for s in range(nbatch_e2e):
        ns, H, O = batches[s]
        hH = [h.cpu().pin_memory() for h in H]
        hO = [o.cpu().pin_memory() for o in O]
        hw = [torch.empty(n, dtype=torch.float64).pin_memory() for n in ns]
        hout = [torch.empty(ns[k], ns[b], dtype=torch.float64).pin_memory() for b, k in zip(bra, ket)]
        hb.append((ns, hH, hO, hw, hout))
    e2e_steps = max(3, min(args.steps, 8)) if hb else 0
    for s in range(1 if hb else 0):
        ns, hH, hO, hw, hout = hb[0]
        ctx.eig_recalc_step(ns, [x.data_ptr() for x in hH], [x.data_ptr() for x in hw], None, bra, ket,
                            [x.data_ptr() for x in hO], [x.data_ptr() for x in hout])
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        ns, hH, hO, hw, hout = hb[i % len(hb)]
        ctx.eig_recalc_step(ns, [x.data_ptr() for x in hH], [x.data_ptr() for x in hw], None, bra, ket,
                            [x.data_ptr() for x in hO], [x.data_ptr() for x in hout])
    torch.cuda.synchronize()
    e2e_elapsed = max(time.perf_counter() - t0, 1e-9)
    if dist:
        t = torch.tensor([e2e_elapsed], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_elapsed = float(t.item())
    e2e_value = world * 3600.0 / (STEPS_PER_RUN * e2e_elapsed / e2e_steps) if hb else None
    ns0 = batches[0][0]
    h2d = sum(8 * n * n for n in ns0) + sum(8 * ns0[b] * ns0[k] for b, k in zip(bra, ket))
    d2h = sum(8 * n for n in ns0) + sum(8 * ns0[b] * ns0[k] for b, k in zip(bra, ket))
    # ---- roofline of the dominant kernel ----
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
    top = max(kstats.items(), key=lambda kv: kv[1][1])
    name, (nl, ms) = top
    steps_ns = [batches[(args.warmup + i) % nbatch][0] for i in range(args.steps)]
    roof = None
    if name == "gemm_f64":
        name = "gemm_f64"
    if name == "trd_panel" and nl:
        bytes_total = sum(trd_panel_step_bytes(ns) for ns in steps_ns)
        per_launch_bytes = bytes_total / nl
        achieved = per_launch_bytes / (ms / nl / 1000.0) / 1e9
        roof = {"kernel": "trd_panel", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "peak_source": hbm_src + " (MEASURED_PEAKS.json hbm_gbs)", "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": None,
                "launches": nl, "avg_launch_ms": ms / nl,
                "algorithmic_bytes_per_launch": per_launch_bytes}
    elif nl:
        # FP64 contraction: measured DGEMM throughput as the denominator
        peak = fp64_gemm_peak(torch, dev)
        flops = sum(algorithmic_flops(ns) - sum(14.0 / 3.0 * n ** 3 for n in ns) for ns in steps_ns)
        achieved = flops / (ms / 1000.0) / 1e12
        roof = {"kernel": name, "bound": "tensor", "achieved": achieved, "peak": peak,
                "peak_source": "measured cuBLAS DGEMM 8192^3 in this run (FP64 tensor pipe)",
                "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                "launches": nl, "avg_launch_ms": ms / nl}
    share = {k: (v[1] / max(1e-9, sum(x[1] for x in kstats.values()))) for k, v in kstats.items()}
    line = {"metric": METRIC, "value": value, "unit": "runs/hour", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "40-block eigensolve + recalc step (16..4096, log-uniform), 20 steps per run",
                       "blocks_per_step": NBLOCKS, "ops_per_pair": NOPS_PER_PAIR, "steps_per_run": STEPS_PER_RUN,
                       "parallelism": "replicas only" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (%.2f GB of blocks per step)" % (8 * sum(n * n for n in batches[0][0]) / 1e9)},
            "latency_ms": {"step_p50": float(np.percentile(step_ms, 50)), "step_p99": float(np.percentile(step_ms, 99)),
                           "run_p50": float(np.percentile(step_ms, 50)) * STEPS_PER_RUN,
                           "run_p99": float(np.percentile(step_ms, 99)) * STEPS_PER_RUN},
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "runs/hour", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": roof,
            "kernel_time_share": {k: round(v, 4) for k, v in share.items() if v > 0.001},
            "gemm_ms_per_step_by_site": {k: round(v[1] / args.steps, 3) for k, v in gemm_sites.items()}}
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t, frac = cpu_step(0, threads, budget_s=args.cpu_budget)
        cpu_ms = 1000.0 * t / frac
        line["cpu_baseline"] = {"value": 3600.0 / (STEPS_PER_RUN * cpu_ms / 1000.0), "unit": "runs/hour",
                                "cores": threads, "kind": "port",
                                "sample": "one step: blocks with n <= %d in random order until %.0f s of work (dsyev per "
                                          "block over %d threads, BLAS gemm recalc), extrapolated to the whole step by "
                                          "algorithmic flops (%.1f%% of them done)"
                                          % (CPU_SAMPLE_NMAX, args.cpu_budget, threads, 100 * frac)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ncu_small(nmax):
    """Small profiling case (no torch on the GPU): 12 blocks with sizes up to
    `nmax` and their 72 operators through the host-buffer C ABI, twice."""
    import nrgb
    rng = np.random.default_rng(SEED)
    ns = [int(x) for x in np.linspace(48, nmax, 12)]
    bra = [k for k in range(len(ns)) for _ in range(NOPS_PER_PAIR)]
    ket = [(k + 1) % len(ns) for k in range(len(ns)) for _ in range(NOPS_PER_PAIR)]
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
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=4.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    ap.add_argument("--nmax", type=int, default=4096, help="cap on block sizes (small profiling cases)")
    ap.add_argument("--ncu-small", type=int, default=0,
                    help="run only the small profiling case with blocks up to this size (no torch GPU work)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global NMAX
    NMAX = args.nmax
    if args.ncu_small:
        return run_ncu_small(args.ncu_small)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world)


if __name__ == "__main__":
    sys.exit(main())
