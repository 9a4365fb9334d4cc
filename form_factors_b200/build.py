"""Builds libffb200.so in-tree with nvcc for sm_100a.

Floating-point flags are part of the contract: --fmad=false (no FMA
contraction), IEEE division and square root (-prec-div=true -prec-sqrt=true),
no fast-math, host code with -ffp-contract=off.  Hit indices and points are
bit-identical to the reference's CPU casters only under these flags.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libffb200.so")
PROBE_LIB = os.path.join(PKG, "libffb200_probe.so")

CUDA_SOURCES = ["ffb_api.cu", "ffb_static.cu"]
CXX_SOURCES = ["ffb_systems.cpp", "ffb_server.cpp", "ffb_thermal.cpp", "ffb_host_rows.cpp"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
    "--expt-relaxed-constexpr",
]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libffb200.so")
    return cand


def sources():
    return [os.path.join(CSRC, s) for s in CUDA_SOURCES + CXX_SOURCES]


def deps():
    out = sources()
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in deps())


def build_probe(force=False, verbose=False):
    """libffb200_probe.so: the FP32 issue-rate probe bench.py uses as a peak."""
    src = os.path.join(CSRC, "ffb_probe.cu")
    if not force and os.path.exists(PROBE_LIB) and os.path.getmtime(PROBE_LIB) >= os.path.getmtime(src):
        return PROBE_LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-shared", src, "-o", PROBE_LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(PROBE_LIB + ".tmp", PROBE_LIB)
    return PROBE_LIB


def build(force=False, verbose=False, ptxas_verbose=False):
    """Compiles libffb200.so (and the probe) unless newer than every source."""
    build_probe(force, verbose)
    if not force and up_to_date():
        return LIB
    obj_dir = os.path.join(PKG, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    for src in sources():
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + extra + ["-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc()] + NVCC_FLAGS + ["-x", "c++", "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="--ptxas-v" in sys.argv)
