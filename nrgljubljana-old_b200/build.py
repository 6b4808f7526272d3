"""Build libnrgb.so in-tree for sm_100a (nvcc for .cu, g++ via nvcc for .cc).

    python nrgljubljana-old_b200/build.py [--force]

Outputs nrgljubljana-old_b200/libnrgb.so.  Object files go to
nrgljubljana-old_b200/_build/.  Rebuilds only what changed."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnrgb.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I" + os.path.join(ROOT, "include")]


def sources():
    out = []
    for sub in ("csrc", "host"):
        d = os.path.join(HERE, sub)
        for f in sorted(os.listdir(d)):
            if f.endswith((".cu", ".cc")):
                out.append(os.path.join(d, f))
    return out


def headers():
    hs = [os.path.join(ROOT, "include", "nrgb.h")]
    for sub in ("csrc", "host"):
        d = os.path.join(HERE, sub)
        hs += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return hs


def build(force=False, verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    hmax = max(os.path.getmtime(h) for h in headers())
    objs = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hmax):
            continue
        cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
        if src.endswith(".cc"):
            cmd = [NVCC] + COMMON + ["-x", "cu", "-c", src, "-o", obj] + ARCH
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcuda"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
