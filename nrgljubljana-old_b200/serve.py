"""Serving workload: a stream of NRG runs through the run server.

The stream is the z-averaging / parameter-sweep workload of a served NRG
deployment: single-impurity Anderson model, QS symmetry, flat band,
U = 0.2, Gamma = 0.02, Lambda = 2, Nmax = 40, FDM spectral function
A(omega) of the impurity level at T = 1e-6 with 50 bins per decade; Nz = 8
z-shifts (z = k/8, k = 1..8) crossed with 32 values of eps_d drawn (seeded)
uniformly from [-0.2, 0]; Nkeep of each run drawn (seeded) uniformly from
{200, 500, 1000, 2000}.  Requests arrive as a Poisson process at a stated
rate (rate 0: all at once, which measures capacity).

The reference has no serving layer: one `nrg` process per run
(src/nrg.cc:3429-3469).  The plain path here is nrgb_run on one context,
one run after another.
"""
import os
import threading
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

import inputgen
import nrgb

U, GAMMA, LAMBDA, NMAX, T_FDM = 0.2, 0.02, 2.0, 40, 1e-6
KEEPS = (200, 500, 1000, 2000)
SEED = 20261208


@dataclass
class Request:
    z: float
    eps_d: float
    keep: int
    workdir: str = ""
    outdir: str = ""


def stream(n_z: int = 8, n_eps: int = 32, seed: int = SEED) -> List[Request]:
    """The seeded request list in arrival order (eps_d runs fastest)."""
    rng = np.random.default_rng(seed)
    eps = rng.uniform(-0.2, 0.0, n_eps)
    keeps = rng.choice(np.array(KEEPS), size=n_z * n_eps)
    out = []
    for k in range(n_z):
        for e in range(n_eps):
            out.append(Request(z=(k + 1) / n_z, eps_d=float(eps[e]), keep=int(keeps[k * n_eps + e])))
    return out


def params(keep: int) -> Dict[str, object]:
    return {"keep": keep, "fdm": True, "T": T_FDM, "specd": "A_d-A_d", "bins": 50,
            "savebins": True, "broaden": False}


def prepare(reqs: List[Request], root: str) -> List[Request]:
    """Write each request's param/data (the input files of one run)."""
    for i, r in enumerate(reqs):
        r.workdir = os.path.join(root, "in%04d" % i)
        r.outdir = os.path.join(root, "out%04d" % i)
        os.makedirs(r.outdir, exist_ok=True)
        inputgen.make_siam(r.workdir, U, r.eps_d, GAMMA, LAMBDA, NMAX, z=r.z, params=params(r.keep))
    return reqs


def arrivals(n: int, rate_hz: float, seed: int = SEED + 1) -> np.ndarray:
    """Poisson arrival offsets (s) of n requests; rate 0 -> all at t = 0."""
    if rate_hz <= 0:
        return np.zeros(n)
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_hz, n)) - 0.0


def serve(server: "nrgb.Server", reqs: List[Request], rate_hz: float, seed: int = SEED + 1,
          timeout_s: float = 3600.0) -> Dict[str, object]:
    """Submit `reqs` at Poisson arrival times and wait for all of them.
    Returns the per-run statistics and the stream summary."""
    offs = arrivals(len(reqs), rate_hz, seed)
    tickets: List[Optional[int]] = [None] * len(reqs)
    t_sub = [0.0] * len(reqs)
    err: List[BaseException] = []

    def submitter():
        try:
            t0 = time.perf_counter()
            for i, r in enumerate(reqs):
                d = t0 + offs[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                t_sub[i] = time.perf_counter()
                tickets[i] = server.submit(r.workdir, r.outdir)
        except BaseException as e:  # surfaced by the caller
            err.append(e)

    t_start = time.perf_counter()
    th = threading.Thread(target=submitter)
    th.start()
    runs = [None] * len(reqs)
    t_done = [0.0] * len(reqs)
    readback = 0
    for i in range(len(reqs)):
        while tickets[i] is None and not err:
            time.sleep(0.0005)
        if err:
            break
        runs[i] = server.wait(tickets[i], timeout_s)
        t_done[i] = t_sub[i] + runs[i]["latency_s"]
        # the client reads its result back: thermodynamics and the spectrum
        for name in os.listdir(reqs[i].outdir):
            with open(os.path.join(reqs[i].outdir, name), "rb") as fh:
                readback += len(fh.read())
    t_client = time.perf_counter()
    th.join()
    if err:
        raise err[0]
    t_end = max(t_done)
    lat = np.array([r["latency_s"] for r in runs])
    span = t_end - t_start
    return {
        "runs": runs,
        "n": len(reqs),
        "span_s": span,
        "runs_per_hour": 3600.0 * len(reqs) / span,
        "client_span_s": t_client - t_start,
        "client_runs_per_hour": 3600.0 * len(reqs) / (t_client - t_start),
        "readback_bytes": readback,
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_queue_s": float(np.mean([r["queue_s"] for r in runs])),
        "counters": server.counters(),
        "rate_hz": rate_hz,
    }


def plain(reqs: List[Request], device: int = 0, per_block: bool = False) -> Dict[str, object]:
    """The plain FP64 path: nrgb_run on one context, one run after another;
    per_block=True makes one eigensolver call per block (the reference's
    per-subspace dsyev structure) instead of one batched call per step."""
    ctx = nrgb.Context(device)
    try:
        if per_block:
            ctx.set_eig_mode(1)
        t0 = time.perf_counter()
        stats = [ctx.run(r.workdir, r.outdir) for r in reqs]
        span = time.perf_counter() - t0
    finally:
        ctx.close()
    return {"runs": stats, "n": len(reqs), "span_s": span, "runs_per_hour": 3600.0 * len(reqs) / span,
            "per_keep_s": {k: float(np.mean([s["wall_s"] for s, r in zip(stats, reqs) if r.keep == k]))
                           for k in sorted({r.keep for r in reqs})}}
