"""Build libfdcuda.so in-tree: the CUDA perturbation route for sm_100a plus its C++ host.

    python -m fractodactyl_b200.build [--verbose]

Flags that matter for parity: -fmad=false on the plain-form kernels and
-ffp-contract=off on host code, so no a*b+c is fused (the reference's Rust never
fuses); the precision-form kernels keep fused multiply-adds.
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfdcuda.so")
BUILD = os.path.join(HERE, "_build")
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]))
    return r


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)) + [
        os.path.join(os.path.dirname(HERE), "include", f) for f in ("fdcuda.h", "fdhost.h")]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(verbose=False, force=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    cxx = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"]
    objs = []
    host_o = os.path.join(BUILD, "host.o")
    run(cxx + ["-c", os.path.join(CSRC, "host.cpp"), "-o", host_o], verbose)
    objs.append(host_o)
    common = [nvcc(), ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-Xptxas", "-v" if verbose else "-O3"]
    for src, fmad in (("fdcuda.cu", "false"), ("peaks.cu", "false"), ("perturb_f32.cu", "true"), ("noalloc.cu", "false")):
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        run(common + ["-fmad=" + fmad, "-c", path, "-o", o], verbose)
        objs.append(o)
    tmp = OUT + ".tmp"
    run([nvcc(), ARCH, "-shared", "-o", tmp] + objs + ["-lpthread"], verbose)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force or a.verbose))
