"""Build libshg_b200.so (the C-ABI library of include/shg.h) in-tree for sm_100a.

    python -m cushg_b200.build [--force]

Every .cu under cushg_b200/csrc is compiled by nvcc for `arch=compute_100a,code=sm_100a`
into an object under cushg_b200/_objs/ and linked into cushg_b200/libshg_b200.so; the
command-line drop-in csrc/cli/cushg_main.cpp links against it as cushg_b200/cushg.
Objects are rebuilt only when their sources or headers changed; independent objects
compile in parallel.
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
OBJ = os.path.join(PKG, "_objs")
LIB = os.path.join(PKG, "libshg_b200.so")
CLI = os.path.join(PKG, "cushg")
CLI_SRC = os.path.join(CSRC, "cli", "cushg_main.cpp")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I", os.path.join(ROOT, "include")]


def _cuda_root() -> str:
    """The CUDA toolkit that holds nvcc (its include/ and lib64/ serve the command-line tool)."""
    nvcc = shutil.which(NVCC) or "/usr/local/cuda/bin/nvcc"
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "shg.h")]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if force or _stale(CLI, [CLI_SRC, LIB, os.path.join(ROOT, "include", "shg.h")]):
        cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
        cuda = _cuda_root()
        cmd = [cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
               CLI_SRC, "-o", CLI, "-L", PKG, "-lshg_b200", "-L", os.path.join(cuda, "lib64"), "-lcudart",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built", LIB, "and", CLI)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(force=a.force, verbose=True)
    sys.exit(0)
