#!/usr/bin/env python3
"""Build libfrb200.so in-tree (sm_100a only).

    python hifiles-solver_b200/build.py [--force] [--verbose]

The library holds the host set-up (C++), the fused FR stage kernels and the
per-operator kernels behind the C ABI of include/fr_b200.h.  nvcc cross-compiles
for sm_100a, so this runs on a machine without a GPU.
"""
import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libfrb200.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = ["fr_host.cpp", "fr_restart.cpp", "fr_vtu.cpp", "fr_solver.cu", "fr_ops.cu", "fr_noalloc.cu", "fr_runner_quad_f64.cu",
           "fr_runner_quad_f32.cu", "fr_runner_hex_f64_a.cu", "fr_runner_hex_f64_p3.cu", "fr_runner_hex_f64_p4.cu",
           "fr_runner_hex_f32.cu", "fr_mlp.cu", "fr_diag.cu", "fr_tc_gemm.cu", "fr_mixed.cpp", "fr_batch_merged.cu", "fr_mixed_fused.cu",
           "fr_mixed_fused_2d.cu", "fr_mixed_fused_p14.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _newer(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h", ".inc"))]
    headers.append(os.path.join(REPO, "include", "fr_b200.h"))
    objs = []
    procs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if not force and not _newer(obj, [path] + headers):
            continue
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
               "-I", os.path.join(REPO, "include"), "-I", CSRC, "-c", path, "-o", obj]
        if src.endswith(".cu"):
            # reference rounding: no implicit contraction of a*b+c into an FMA
            cmd[1:1] = ["-fmad=false"] + (["-Xptxas", "-v"] if verbose else [])
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stdout.write(out)
        if p.returncode != 0:
            failed = True
            print("build failed:", src)
    if failed:
        raise SystemExit(1)
    if force or procs or not os.path.exists(OUT):
        cmd = [NVCC, *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
