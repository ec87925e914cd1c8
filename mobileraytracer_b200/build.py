"""Build libmrt_cuda.so in-tree for sm_100a (B200).

    python -m mobileraytracer_b200.build [--verbose] [--ptxas-info]

Flags that matter for parity: --fmad=false (no FMA contraction), -prec-div=true, -prec-sqrt=true,
-ftz=false (IEEE division / square root, denormals kept), and -ffp-contract=off for the host
compiler, so the device arithmetic rounds like the reference's compiled C++.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
OUT = os.path.join(OUT_DIR, "libmrt_cuda.so")
SOURCES = ["mrt_capi.cu", "mrt_bvh.cu", "mrt_grid.cu", "mrt_kernels.cu", "mrt_render.cu", "mrt_batch.cu", "mrt_obj.cu",
           "mrt_raster.cu", "mrt_serve.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "-ccbin", "/usr/bin/g++",
]


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "mrt_cuda.h"), os.path.abspath(__file__)]
    if not force and os.path.exists(OUT) and not ptxas_info:
        built = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= built for d in deps):
            return OUT
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        cmd = [NVCC, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if out and (verbose or ptxas_info or p.returncode):
            print(out, file=sys.stderr)
        if p.returncode:
            failed = True
    if failed:
        raise RuntimeError("nvcc failed")
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-ccbin", "/usr/bin/g++", *objs, "-o", OUT]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    for o in objs:
        os.remove(o)
    return OUT


DROPIN_SRC = os.path.join(HERE, "cpp", "src", "dropin.cpp")
DROPIN_OUT = os.path.join(OUT_DIR, "libmrt_dropin.so")


def build_dropin(verbose: bool = False, force: bool = False) -> str:
    """libmrt_dropin.so: the MobileRT C++ API (cpp/include) over libmrt_cuda.so."""
    lib = build(verbose=verbose)
    deps = [DROPIN_SRC, lib, os.path.join(HERE, "cpp", "include", "MobileRT", "b200_api.hpp")]
    if not force and os.path.exists(DROPIN_OUT) and all(os.path.getmtime(d) <= os.path.getmtime(DROPIN_OUT) for d in deps):
        return DROPIN_OUT
    cmd = ["/usr/bin/g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-I", os.path.join(HERE, "cpp", "include"), "-I", os.path.join(HERE, "cpp", "glm_min"),
           DROPIN_SRC, "-L", OUT_DIR, "-lmrt_cuda", "-Wl,-rpath,$ORIGIN", "-o", DROPIN_OUT]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return DROPIN_OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_info, a.force or a.ptxas_info))
    print(build_dropin(a.verbose, a.force))
