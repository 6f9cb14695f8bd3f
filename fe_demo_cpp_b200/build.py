"""Build libfem_b200.so in-tree for sm_100a (nvcc, no torch extension API).

    python -m fe_demo_cpp_b200.build [--force] [--verbose]

Objects go to fe_demo_cpp_b200/_build/, the library to
fe_demo_cpp_b200/lib/libfem_b200.so (both git-ignored; the .so travels with
the working tree).  Sources are compiled in parallel; a rebuild happens only
when a source or header is newer than the library.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libfem_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home() -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _compile(src: str, verbose: bool, ptxas_v: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    inc = ["-I", INCLUDE, "-I", CSRC]
    if src.endswith(".cu"):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *inc, "-c", src, "-o", obj]
        if ptxas_v:
            cmd[1:1] = ["-Xptxas", "-v"]
    else:
        cmd = ["g++", *CXX_FLAGS, *inc, "-I", os.path.join(cuda_home(), "include"), "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{res.stdout}\n{res.stderr}")
    if verbose or ptxas_v:
        out = (res.stdout + res.stderr).strip()
        if out:
            print(out, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    srcs = sources()
    if not force and os.path.exists(LIB):
        t_lib = os.path.getmtime(LIB)
        if all(os.path.getmtime(f) <= t_lib for f in srcs + headers()):
            return LIB
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, ptxas_v), srcs))
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed\n{res.stdout}\n{res.stderr}")
    os.replace(LIB + ".tmp", LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print registers / spills / smem per kernel")
    a = ap.parse_args(argv)
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose, ptxas_v=a.ptxas_v))


if __name__ == "__main__":
    sys.exit(main())
