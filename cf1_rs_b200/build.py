"""Build recipe for the sm_100a library (libcf1gpu.so) and the synthetic-input
library (libcf1synth.so), both in-tree under cf1_rs_b200/.

    python -m cf1_rs_b200.build          # or __graft_entry__.build()
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcf1gpu.so")
SYNTH_LIB = os.path.join(HERE, "libcf1synth.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
           "-Xptxas", "-v", "--expt-relaxed-constexpr"] + ARCH

SOURCES = [
    "cf1_util.cu",
    "cf1_phase12.cu",
    "cf1_phase3_sort.cu",
    "cf1_msdsort.cu",
    "cf1_bbhash.cu",
    "cf1_learned.cu",
    "cf1_phase4.cu",
    "cf1_pipeline.cu",
    "cf1_export.cu",
    "cf1_fasta.cu",
    "cf1_capi.cu",
    "cf1_noalloc.cu",
    "cf1_tuner.cu",
    "cf1_binfile.cu",
]
HEADERS = [f for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] if os.path.isdir(CSRC) else []


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "cf1gpu.h")]
    if _newer(obj, deps):
        return obj
    log = os.path.join(BUILD, os.path.splitext(src)[0] + ".ptxas.log")
    cmd = [NVCC] + NVFLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    with open(log, "w") as f:
        r = subprocess.run(cmd, stdout=f, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        sys.stderr.write(open(log).read())
        raise RuntimeError(f"nvcc failed on {src} (see {log})")
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    if not _newer(LIB, objs):
        cmd = [NVCC, "-shared"] + ARCH + ["-o", LIB] + objs + ["-lz"]
        subprocess.run(cmd, check=True)
    synth_src = os.path.join(CSRC, "cf1_synth.cpp")
    if os.path.exists(synth_src) and not _newer(SYNTH_LIB, [synth_src]):
        subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-Wall", "-o", SYNTH_LIB,
                        synth_src], check=True)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
