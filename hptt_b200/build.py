"""Build libhptt_cuda.so in-tree for sm_100a with nvcc, and libhptt.so (the
C++14 hptt::create_plan interface of include/hptt/hptt.h) over it with g++.

    python -m hptt_b200.build            # incremental
    python -m hptt_b200.build --clean    # from scratch

Objects go to hptt_b200/_build/ (git-ignored); the shared library is written
next to this file so it travels with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhptt_cuda.so")
CXX_SRC = os.path.join(HERE, "cxx")
LIB_CXX = os.path.join(HERE, "libhptt.so")
CXX = os.environ.get("CXX", "g++")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-I", CSRC, "-I", INCLUDE]
CU_FLAGS = ARCH + COMMON + ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, name))
    return out


def _headers_mtime():
    m = 0.0
    for d in (CSRC, INCLUDE):
        for root, _, files in os.walk(d):
            for f in files:
                if f.endswith((".h", ".cuh")):
                    m = max(m, os.path.getmtime(os.path.join(root, f)))
    return m


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    hdr = _headers_mtime()
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr):
        return obj
    flags = CU_FLAGS if src.endswith(".cu") else ARCH + COMMON + ["-x", "cu"]
    cmd = [NVCC] + flags + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed on {src}")
    if verbose and r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(clean: bool = False, verbose: bool = False) -> str:
    if clean and os.path.isdir(BUILD):
        shutil.rmtree(BUILD)
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcublas"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    build_cxx(verbose)
    return LIB


def build_cxx(verbose: bool = False) -> str:
    """libhptt.so: hptt::create_plan and the create_trans_plan_impl_* factories
    (C++14), linked against libhptt_cuda.so next to it."""
    srcs = [os.path.join(CXX_SRC, f) for f in sorted(os.listdir(CXX_SRC)) if f.endswith(".cpp")]
    deps = srcs + [LIB]
    for root, _, files in os.walk(INCLUDE):
        deps += [os.path.join(root, f) for f in files if f.endswith(".h")]
    if os.path.exists(LIB_CXX) and os.path.getmtime(LIB_CXX) >= max(os.path.getmtime(d) for d in deps):
        return LIB_CXX
    cmd = [CXX, "-std=c++14", "-O2", "-fPIC", "-shared", "-Wall", "-I", INCLUDE] + srcs + \
          ["-o", LIB_CXX, "-L", HERE, "-lhptt_cuda", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("g++ failed on the C++ interface")
    return LIB_CXX


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(clean=a.clean, verbose=a.verbose))


if __name__ == "__main__":
    main()
