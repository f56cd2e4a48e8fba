"""Build recipe for the sm_100a library (libhn_sm100.so) and its host C++ layer.

Compiles every CUDA source under csrc/ with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a), links one shared library in-tree
next to this file, and builds the host C++ solver library (libhn_host.so)
that sits above the C ABI. Run `python build.py` or call build().
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhn_sm100.so")
HOSTLIB = os.path.join(HERE, "libhn_host.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: every a*b+c rounds the product and the sum separately, as the
# reference's x86-64 build does, so elementwise results match it bit for bit.
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
           "-I", INCLUDE, "-I", CSRC]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_cuda(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(INCLUDE, "hn_sm100.h")]
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers) or ptxas_info:
            cmd = [NVCC, *ARCH, *NVFLAGS, "-c", src, "-o", obj]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    return LIB


def build_host(verbose: bool = False) -> str | None:
    """Host C++ layer: each source compiled separately (the dense LDL^T may
    contract to FMA; the IPM's scalar arithmetic must not, to match the
    reference's rounding), then linked against libhn_sm100.so."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if not srcs:
        return None
    hdrs = glob.glob(os.path.join(HOST, "*.hpp")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else os.environ.get("CXX", "g++")
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    for src in srcs:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            contract = "-ffp-contract=fast" if os.path.basename(src) == "hn_ldlt.cpp" else "-ffp-contract=off"
            # the MPS and LP readers look names up by string_view (C++20 heterogeneous lookup)
            std = "-std=c++20" if os.path.basename(src) == "hn_read.cpp" else "-std=c++17"
            cmd = [cxx, "-O3", std, "-fPIC", "-fopenmp", "-march=x86-64-v3", contract,
                   "-I", INCLUDE, "-I", HOST, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if _stale(HOSTLIB, objs + [LIB]):
        _run([cxx, "-shared", "-fopenmp", "-o", HOSTLIB, *objs, "-L", HERE, "-lhn_sm100",
              "-Wl,-rpath,$ORIGIN", "-lpthread"])
    return HOSTLIB


def build(verbose: bool = False) -> None:
    build_cuda(verbose)
    build_host(verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
