"""Builds libsj.so (the engine, sm_100a) and the sj_main CLI in-tree.

Usage: python -m sjoin.build [--force]   (from the package directory), or
       sjoin.build.build() from Python.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)                 # self-join-hpbdc2019_b200/
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libsj.so")
CLI = os.path.join(PKG, "sj_main")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["sj_prims.cu", "sj_index.cu", "sj_stencil.cu", "sj_tasks.cu", "sj_join.cu", "sj_emit.cu", "sj_estimate.cu"]
CPP_SOURCES = ["sj_api.cpp", "sj_csv.cpp"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if not force and not _newer(obj, [src] + _headers()):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
               "-I", CSRC, "-I", INCLUDE, "-c", src, "-o", obj]
    else:
        cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I", CSRC, "-I", INCLUDE,
               "-I", os.path.join(CUDA, "include"), "-c", src, "-o", obj]
    subprocess.check_call(cmd)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in CU_SOURCES + CPP_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _newer(LIB, objs):
        subprocess.check_call([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", LIB, *objs,
                               "-Xlinker", "--no-undefined", "-lgomp", "-lpthread", "-ldl", "-lrt"])
    cli_src = os.path.join(CSRC, "sj_cli.cpp")
    if os.path.exists(cli_src) and (force or _newer(CLI, [cli_src, LIB] + _headers())):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", INCLUDE, cli_src, "-o", CLI,
                               "-L", PKG, "-lsj", "-Wl,-rpath,$ORIGIN"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
