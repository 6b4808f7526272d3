"""Run the CPU oracle on the full-size workloads of nrg_cases.GOLDEN_CASES and
store their outputs as tests/golden/nrg/<case>.npz, with the sha256 of the
generated `param`/`data` they were made from.

    python tests/golden/make_nrg_goldens.py [case ...] [--threads N] [--driver ev|evd] [--spill]

The oracle diagonalises with LAPACK dsyev by default (the reference's
routine, src/diag.h:54-89); `--driver evd` uses dsyevd, which gives the same
eigenvalues to rounding and is several times faster on blocks of thousands.
Each fixture records the driver and the thread count it was made with.
Blocks are diagonalised concurrently on `--threads` host threads (OpenMP over
blocks in the reference, src/nrg.cc:2484-2507)."""
import argparse
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "nrgljubljana-old_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import nrg_cases as cases  # noqa: E402
import nrg_oracle as O  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--driver", default="ev", choices=("ev", "evd"))
    ap.add_argument("--spill", action="store_true", help="keep eigenvectors on disk (memory-mapped)")
    ap.add_argument("--tmp", default=None, help="directory for the inputs and spilled eigenvectors")
    a = ap.parse_args()
    names = a.cases or sorted(cases.GOLDEN_CASES)
    os.makedirs(os.path.join(HERE, "nrg"), exist_ok=True)
    for name in names:
        with tempfile.TemporaryDirectory(dir=a.tmp) as tmp:
            wd = cases.make_case(name, os.path.join(tmp, "in"))
            out = os.path.join(tmp, "out")
            t0 = time.time()
            spill = None
            if a.spill:
                spill = os.path.join(tmp, "spill")
                os.makedirs(spill)
            o = O.Oracle(wd, threads=a.threads, eigh_driver=a.driver, spill_dir=spill, progress=True)
            o.run(out)
            dt = time.time() - t0
            meta = {"case": name, "driver": a.driver, "threads": a.threads, "seconds": round(dt, 1)}
            cases.save_golden(os.path.join(HERE, "nrg", name + ".npz"), cases.load_outputs(out),
                              cases.input_digest(wd), meta)
            print(name, meta, flush=True)


if __name__ == "__main__":
    main()
