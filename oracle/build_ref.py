"""Builds the reference's own sources into oracle/_ref/ (test / baseline infrastructure).

The reference's sources are compiled where they lie: the directory named by
the SJ_REFERENCE environment variable, else a checkout named `reference` next
to this repository; nothing is copied.  Its dimensions are compile-time macros
in params.h, which every file includes with #include "params.h", so each
configuration gets a directory of symbolic links to the reference files plus a
generated params.h: the compiler resolves quoted includes relative to the
link's directory and therefore picks up that params.h.

Per configuration (GPUNUMDIM, NUMINDEXEDDIM, SORT_BY_WORKLOAD) it produces
  _ref/ref_dump_D{D}_K{k}_S{s}{v}      one reference kernel, single batch, raw pairs
  _ref/ref_pipeline_D{D}_K{k}_S{s}{v}  the reference's batched pipeline, timed
  _ref/ref_import_D{D}                 the reference's CSV import (CPU only)

Variant v = "" is the reference exactly as shipped.  With nvcc 12.9 its device
code finds no grid cell at all: every cell lookup is a thrust::binary_search
whose comparison calls gridCellLookup::operator< (structs.h:91), a host-only
member, so on the device every kernel emits zero pairs (measured on a B200).
Variant v = "_hd" differs in that one declaration only: its structs.h is
generated here from the original with `__host__ __device__` added to that
operator, which is what the device code needs to compare cells.  Every other
file is the original, linked in place.
Flags follow the reference makefile (makefile:13) with the architecture set
to sm_100a.  The reference cannot run without a GPU; the binaries travel to
the GPU box with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
REFERENCE = os.environ.get("SJ_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
REF_FILES = ["GPU.cu", "GPU.h", "import_dataset.cpp", "kernel.cu", "kernel.h", "kernelloops.h", "main.cu",
             "stamploops.h", "stamploopsV2.h", "stamploopsSortingCells.h", "structs.h"]
# (GPUNUMDIM, NUMINDEXEDDIM, SORT_BY_WORKLOAD, variant)
CONFIGS = [(2, 2, 0, ""), (2, 2, 0, "_hd"), (2, 2, 1, "_hd"), (3, 3, 0, "_hd"), (4, 4, 0, "_hd"),
           (6, 6, 0, "_hd"), (16, 6, 0, "_hd"), (5, 3, 0, "_hd")]
HD_FROM = "bool operator<(const gridCellLookup & other) const"
HD_TO = "__host__ __device__ bool operator<(const gridCellLookup & other) const"
FLAGS = ["-std=c++14", "-O3", "-Xcompiler", "-fopenmp", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-D_MWAITXINTRIN_H_INCLUDED", "-D_FORCE_INLINES", "-w"]

PARAMS = """#define BLOCKSIZE 256
#define THREADPERPOINT 1
#define SORT_BY_WORKLOAD {s}
#define GPUNUMDIM {d}
#define NUMINDEXEDDIM {k}
#define DTYPE double
#define NB_THREAD_THIRD1 16
#define NB_THREAD_THIRD2 8
#define NB_THREAD_THIRD3 2
"""


def available() -> bool:
    return all(os.path.exists(os.path.join(REFERENCE, f)) for f in REF_FILES)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("failed: " + " ".join(cmd) + "\n" + r.stderr[-3000:])


def _farm(d, k, s, v="") -> str:
    src = os.path.join(OUT, f"src_D{d}_K{k}_S{s}{v}")
    os.makedirs(src, exist_ok=True)
    for f in REF_FILES:
        link = os.path.join(src, f)
        if v == "_hd" and f == "structs.h":
            text = open(os.path.join(REFERENCE, f)).read()
            if text.count(HD_FROM) != 1:
                raise RuntimeError("structs.h: comparison operator not found")
            text = text.replace(HD_FROM, HD_TO)
            if os.path.islink(link):
                os.remove(link)
            if not os.path.exists(link) or open(link).read() != text:
                with open(link, "w") as fh:
                    fh.write(text)
            continue
        if not os.path.islink(link):
            if os.path.exists(link):
                os.remove(link)
            os.symlink(os.path.join(REFERENCE, f), link)
    p = os.path.join(src, "params.h")
    text = PARAMS.format(d=d, k=k, s=s)
    if not os.path.exists(p) or open(p).read() != text:
        with open(p, "w") as fh:
            fh.write(text)
    return src


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(x) > os.path.getmtime(target) for x in deps)


def build_config(d, k, s, v="", force=False):
    src = _farm(d, k, s, v)
    tag = f"D{d}_K{k}_S{s}{v}"
    objs = {}
    deps = [os.path.join(src, f) for f in REF_FILES] + [os.path.join(src, "params.h")]
    for name, extra in (("kernel.cu", []), ("GPU.cu", []), ("main.cu", ["-Dmain=sjref_reference_main"]),
                        ("import_dataset.cpp", [])):
        o = os.path.join(src, name + ".o")
        if force or _stale(o, deps):
            _run([NVCC, *FLAGS, *extra, "-I", src, "-c", os.path.join(src, name), "-o", o])
        objs[name] = o
    dump = os.path.join(OUT, f"ref_dump_{tag}")
    if force or _stale(dump, deps + [os.path.join(HERE, "ref_dump.cu")]):
        _run([NVCC, *FLAGS, "-I", src, os.path.join(HERE, "ref_dump.cu"), objs["kernel.cu"], objs["main.cu"],
              objs["GPU.cu"], objs["import_dataset.cpp"], "-o", dump, "-lcuda"])
    pipe = os.path.join(OUT, f"ref_pipeline_{tag}")
    if force or _stale(pipe, deps + [os.path.join(HERE, "ref_pipeline.cu")]):
        _run([NVCC, *FLAGS, "-I", src, os.path.join(HERE, "ref_pipeline.cu"), objs["kernel.cu"], objs["main.cu"],
              objs["GPU.cu"], objs["import_dataset.cpp"], "-o", pipe, "-lcuda"])
    imp = os.path.join(OUT, f"ref_import_D{d}")
    if force or _stale(imp, deps + [os.path.join(HERE, "ref_import.cpp")]):
        _run(["g++", "-O2", "-std=c++14", "-I", src, os.path.join(HERE, "ref_import.cpp"),
              os.path.join(src, "import_dataset.cpp"), "-o", imp])
    return tag


def build(force=False, configs=None) -> bool:
    """Builds every configuration; returns False when the reference is absent."""
    if not available():
        return False
    os.makedirs(OUT, exist_ok=True)
    cfgs = configs or CONFIGS
    with cf.ThreadPoolExecutor(max_workers=min(len(cfgs), 4)) as ex:
        list(ex.map(lambda c: build_config(*c, force=force), cfgs))
    return True


def binary(kind: str, d: int, k: int, s: int = 0, variant: str = "_hd") -> str:
    if kind == "import":
        return os.path.join(OUT, f"ref_import_D{d}")
    return os.path.join(OUT, f"ref_{kind}_D{d}_K{k}_S{s}{variant}")


if __name__ == "__main__":
    ok = build(force="--force" in sys.argv)
    print("reference built into", OUT if ok else "(reference sources absent)")
